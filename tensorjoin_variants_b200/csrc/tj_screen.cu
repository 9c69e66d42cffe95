// Certified tensor-core distance screen for sm_100a (tcgen05 + TMEM + TMA).
//
// For every candidate tile pair (128 R rows x 256 S rows) the kernel computes
// p_ij = z_i . w_j with z = bf16/fp16(x), w = bf16/fp16(y) on the 5th-generation
// tensor cores (FP32 accumulation in TMEM), and sorts each pair into
// certainly-in / certainly-out / band with a rigorous error bound:
//
//   D_ij  = ||x_i||^2 + ||y_j||^2 - 2 x_i.y_j                       (exact reals)
//   |x.y - p| <= R_ij = g ||z|| ||w|| + c + ||x-z|| ||y|| + ||z|| ||y-w||
//
// where g bounds the FP32 accumulation of K exact 16-bit products in any order
// (premise: every accumulation step errs by at most 2 ulp of the partial sum,
// g = (K + 64) 2^-22; products of two 16-bit floats are exact in FP32) and c
// covers underflow.  The reference's FP16 screen uses the same decomposition
// (fp16_gpu_control_20260907/NUMERICAL_SCOPE.md:25-41; epilogue
// two_gate_campaign_20260908/src/gpu_kernels.py:55-88) with an inherited cuBLAS
// premise; here the kernel owns its accumulation, so the premise is stated for
// tcgen05 and checked by the screen-error diagnostics.
//
// Fast path (every pair): v = fma(-2, p, B~_j) in FP32 (two pairs per packed FP32x2 FMA) folded by
// three-input mins per 8-column group, and one compare of each group minimum against a
// per-(row, S tile) threshold tau_i that absorbs every error term; v > tau_i proves the FP64
// oracle value exceeds T.  Groups that pass get per-pair masks: certified FP32 accept, else a
// per-pair FP64 certificate: accept (emit), reject, or band (queued for the FP64 refinement that
// reproduces the oracle's summation order).
//
// Two forms of the same kernel (512 threads, one CTA per SM, persistent over the chunk list):
//   one SM (kPair = false): an item is a 128-row R tile x 256-row S tile, issued as two 128-column
//           half-items (M = 128, N = 128 UMMA) into four TMEM accumulators of 128 columns; half-item
//           s = 2 item + h goes to accumulator s mod 4 and to epilogue group s mod 3, so the three
//           groups work on different half-items at once and the MMA can run up to two items ahead
//   CTA pair (kPair = true, cta_group::2, clusters of 2 SMs, dense single joins with rows of
//           >= 256 elements): an item is a 256 x 256 tile; each CTA loads its 128 A rows and its
//           128-row half of B, CTA 0 issues M = 256 UMMAs into both CTAs' TMEM (2 accumulators of
//           256 columns), stage and accumulator barriers are signalled to both CTAs (tcgen05.commit
//           multicast) and the epilogue warps of both CTAs release accumulators on CTA 0's barrier
//
// Warp roles:
//   warp 0: TMA producer (one lane): a ring of k-block stages and a ring of per-item column-metadata
//           blocks (one 8 KB bulk copy per S tile), so the epilogue never waits on global memory
//   warp 1: TMEM allocator + UMMA issuer (one lane; in the pair, CTA 0's)
//   warps 4-15: epilogue, warp w reads TMEM lanes 32*(w%4) .. +31 (one R row per thread); one SM:
//           group (w-4)/4 takes whole half-items (4 blocks of 32 columns); pair: column thirds of every
//           item (blocks [0,3), [3,6), [6,8)).  Warps synchronise only through mbarriers.
//   warps 2-3: idle (they complete the first warpgroup)
#include <cstddef>
#include <algorithm>
#include <cstring>

#include "tj_emit.cuh"
#include "tj_internal.h"

namespace tj {

namespace {

constexpr int kAccMax = 4;   // TMEM accumulators: one-SM kernel 4 x 128 columns, CTA pair 2 x 256
constexpr int kEpiWarps = 12;                       // three per TMEM lane quarter (column thirds)
constexpr int kEpiFirst = 4;                         // warps 0-3: TMA producer, UMMA issuer, two idle
constexpr int kScreenThreads = (kEpiFirst + kEpiWarps) * 32;
constexpr unsigned kABytes = kTileR * 128;          // 16 KB
constexpr unsigned kBBytes = kTileS * 128;          // 32 KB
constexpr int kMetaSlots = 8;   // items of column metadata in flight (each epilogue group sees several)
constexpr unsigned kDirectMax = 2;   // emission: parts whose lanes hold at most this many pairs each write per lane

// Stage = one 64-element k-block of A (128 rows) and B (256 rows); with the hi/lo split the
// stage holds both limbs of both operands: [A_hi | A_lo | B_hi | B_lo].
template <int kSplit> struct StageCfg {
    static constexpr unsigned kBytes = (kSplit ? 2u : 1u) * (kABytes + kBBytes);   // 48 or 96 KB
    static constexpr int kStages = kSplit ? 2 : 4;
    static constexpr unsigned kAlo = kABytes;                    // offsets inside a split stage
    static constexpr unsigned kBhi = kSplit ? 2u * kABytes : kABytes;
    static constexpr unsigned kBlo = 2u * kABytes + kBBytes;
};

// Column metadata of one S tile (256 sorted rows), structure of arrays.  The screen copies only the
// leading part (ColMetaHot: what its epilogue reads) into shared memory, one bulk copy per item; the
// per-column bounds after it are read from global memory by the screen-error diagnostics.
struct ColMetaHot {
    float nrm2f[kTileS];   // FP32 nearest of ||y - c||^2; +inf for rows beyond the tile's points
    uint32_t perm[kTileS]; // original row id
    float gminB[kTileS / 8];   // per 8-column group: min of nrm2f (the group-wise fast test)
    float WJ, FJ, YJ, BJ, betaJ, WlJ;   // tile maxima of zn, en, yn, nrm2f, |nrm2f - nrm2| bound, zl
    uint32_t c0, nvJ;      // first sorted row, rows that are real points
};
static_assert(sizeof(ColMetaHot) % 16 == 0, "bulk copies need 16-byte multiples");
static_assert(offsetof(ColMetaHot, gminB) % 16 == 0, "group minima are read four at a time");
struct ColMetaF : ColMetaHot {
    float zn[kTileS];      // >= ||w||
    float en[kTileS];      // >= ||y - c - w||
    float yn[kTileS];      // >= ||y - c||
    float zl[kTileS];      // >= ||w_lo||
    double nrm2[kTileS];   // ||y - c||^2 (FP64)
};
static_assert(sizeof(ColMetaF) % 16 == 0 && sizeof(ColMetaHot) % 16 == 0, "16-byte aligned parts");

template <int kStages>
struct ScreenCtl {
    uint64_t full[kStages];
    uint64_t empty[kStages];
    uint64_t acc_full[kAccMax];
    uint64_t acc_empty[kAccMax];
    uint64_t meta_full[kMetaSlots];
    uint64_t meta_empty[kMetaSlots];
    uint64_t drain;
    uint64_t cfull[4];          // one SM: chunk ring (the producer takes chunks from the device queue)
    uint64_t cempty[4];
    unsigned cring[4];
    unsigned tmem_base;
    int abort_flag;
};
constexpr int kChunkRing = 4;
// Stall accounting (TJ_FLAG_SCREEN_TIMES): slots of ScreenArgs::role_t
enum RoleSlot {
    kRoleProd = 0, kRoleProdStage, kRoleProdMeta,
    kRoleMma, kRoleMmaOperand, kRoleMmaAcc,
    kRoleEpi, kRoleEpiMeta, kRoleEpiAcc, kRoleEpiTest, kRoleEpiEmit, kRoleEpiReserve,
    kRoleSlots = 16
};
constexpr unsigned kNoChunk = 0xFFFFFFFFu;

// CTA pair (cta_group::2, 256 x 256 tile over two SMs): a stage holds this CTA's 128 A rows and its
// 128-row half of B for one 64-element k-block; the pair's MMA reads A and B from both CTAs.
struct StageCfgPair {
    static constexpr unsigned kBytes = kABytes + kABytes;   // 32 KB
    static constexpr int kStages = 6;
    static constexpr unsigned kAlo = 0;
    static constexpr unsigned kBhi = kABytes;
    static constexpr unsigned kBlo = 0;
};
template <int kSplit, bool kPair> struct StageSel { using type = StageCfg<kSplit>; };
template <> struct StageSel<0, true> { using type = StageCfgPair; };

template <int kSplit, bool kPair>
constexpr size_t screen_smem() {
    using Cfg = typename StageSel<kSplit, kPair>::type;
    return 1024 + (size_t)Cfg::kStages * Cfg::kBytes + (size_t)kMetaSlots * sizeof(ColMetaHot) +
           sizeof(ScreenCtl<Cfg::kStages>);
}
static_assert(screen_smem<0, false>() <= 232448 && screen_smem<1, false>() <= 232448 &&
              screen_smem<0, true>() <= 232448, "227 KB of shared memory per CTA at most");

// Per-class pointers (a class = joins with the same d, one concatenated operand matrix per side).
struct ScreenClassArgs {
    const uint32_t* r_emit;   // id written into keys for each sorted R row
    const double* r_nrm2;
    const float* r_zn;
    const float* r_en;
    const float* r_zl;
    int kblocks;              // kpad / kbk
    int kpad;                 // operand row length (16, 32 or a multiple of 64 elements)
    int kbk;                  // elements per k-block: 16, 32 or 64 (32-, 64- or 128-byte swizzle)
    unsigned tx_bytes;        // bytes one stage receives for this class (CTA pair)
    unsigned tx_a, tx_h;      // one SM: bytes of a stage's A part and of one 128-row B half (with the split)
    uint32_t desc_hi;         // upper half of the UMMA shared-memory descriptors
};

struct TMaps {
    CUtensorMap a[kMaxClass];
    CUtensorMap b[kMaxClass];
};

struct ScreenArgs {
    const uint4* chunks;       // (global R tile, jlist begin, jlist end, 0)
    const uint32_t* nchunks;   // device count
    const uint32_t* jlist;     // global S tile ids
    const uint4* rtiles;       // (row0 in class operand, nvalid, join, class) per global R tile
    const uint4* stiles;       // same per global S tile
    const ColMetaF* s_meta;    // per global S tile
    const JoinParams* jps;     // per join
    ScreenClassArgs cls[kMaxClass];
    int ncls;
    unsigned idesc;
    // CTA-pair mode: every (R tile, S tile) pair is a candidate; chunks are generated from the grid
    unsigned idesc_pair;       // M = 256 instruction descriptor
    unsigned ntR, ntS, nT;     // R tiles, S tiles, R tile pairs
    uint64_t* acc;
    unsigned long long acc_cap;
    uint64_t* band;
    unsigned long long band_cap;
    Counters* ctr;
    // diagnostics: tile pairs with jlist index % dump_every == 0 write their accumulators (p values)
    float* dump;               // [dump_items][128][256], null when off
    uint4* dump_ids;           // [dump_items]: (global R tile, global S tile, 1, 0)
    unsigned dump_every;
    unsigned dump_items;
    unsigned long long wait_ns;   // limit of every pipeline wait (drains keep kDrainLimitNs)
    // TJ_FLAG_SCREEN_TIMES: %globaltimer of each join's first chunk start (join_t[j], atomicMin) and
    // last chunk end (join_t[njoins + j], atomicMax), and each CTA's start and end (cta_t[2 b], [2 b + 1])
    unsigned long long* join_t;
    unsigned long long* cta_t;
    unsigned long long* role_t;   // [kRoleSlots] SM clock cycles per role and wait, summed over CTAs
    unsigned njoins;
    int nstages;                  // operand stages in the ring (<= the compiled count; a tuning knob)
    int half;                     // one SM: jlist entries carry live-half masks in bits 30-31
};

// One SM: the producer publishes the chunks it takes from the queue in a ring of kChunkRing slots;
// the UMMA issuer and every epilogue warp read them in the same order (kNoChunk ends the sequence).
// Its waits are bounded like every other pipeline wait.
template <int kStages>
TJ_DEV bool publish_chunk(ScreenCtl<kStages>* ctl, unsigned long long q, unsigned c, unsigned long long* status,
                          unsigned long long wait_ns) {
    const unsigned slot = (unsigned)(q % kChunkRing), ph = (unsigned)((q / kChunkRing) & 1);
    if (!mbar_wait(&ctl->cempty[slot], ph ^ 1u, status, wait_ns)) return false;
    *(volatile unsigned*)&ctl->cring[slot] = c;
    mbar_arrive(&ctl->cfull[slot]);   // release: the slot's value is visible to every reader
    return true;
}
// warp-collective in the epilogue warps (every lane reads; lane 0 frees the slot), one lane elsewhere
template <int kStages>
TJ_DEV bool take_chunk(ScreenCtl<kStages>* ctl, unsigned long long q, unsigned& c, unsigned long long* status,
                       unsigned long long wait_ns, bool warp_collective) {
    const unsigned slot = (unsigned)(q % kChunkRing), ph = (unsigned)((q / kChunkRing) & 1);
    bool got = mbar_wait(&ctl->cfull[slot], ph, status, wait_ns);
    if (warp_collective) got = __all_sync(0xffffffffu, got);
    if (!got) return false;
    c = *(volatile unsigned*)&ctl->cring[slot];
    if (warp_collective) __syncwarp();
    if (!warp_collective || lane_id() == 0) mbar_arrive(&ctl->cempty[slot]);
    return true;
}

// Pack the S-side row metadata into one ColMetaF block per 256-row tile.
__global__ void __launch_bounds__(kTileS) build_col_meta(const uint32_t* row0, const uint32_t* nvalid,
                                                          const uint32_t* perm, const double* nrm2,
                                                          const float* nrm2f, const float* zn, const float* en,
                                                          const float* yn, const float* zl, const float* maxZ,
                                                          const float* maxE, const float* maxY, const float* maxB,
                                                          const float* beta, const float* maxZl, ColMetaF* out) {
    const unsigned J = blockIdx.x, t = threadIdx.x;
    const unsigned c0 = row0[J], nv = nvalid[J];
    ColMetaF& m = out[J];
    const bool ok = t < nv;
    const unsigned r = c0 + t;
    m.nrm2f[t] = ok ? nrm2f[r] : INFINITY;
    m.zn[t] = ok ? zn[r] : 0.f;
    m.en[t] = ok ? en[r] : 0.f;
    m.yn[t] = ok ? yn[r] : 0.f;
    m.zl[t] = ok ? zl[r] : 0.f;
    m.perm[t] = ok ? perm[r] : 0u;
    m.nrm2[t] = ok ? nrm2[r] : 0.0;
    float gb = ok ? nrm2f[r] : INFINITY;   // min over the 8 columns t & ~7 .. (t | 7)
    gb = fminf(gb, __shfl_xor_sync(0xffffffffu, gb, 1));
    gb = fminf(gb, __shfl_xor_sync(0xffffffffu, gb, 2));
    gb = fminf(gb, __shfl_xor_sync(0xffffffffu, gb, 4));
    if ((t & 7) == 0) m.gminB[t >> 3] = gb;
    if (t == 0) {
        m.WJ = maxZ[J]; m.FJ = maxE[J]; m.YJ = maxY[J]; m.BJ = maxB[J]; m.betaJ = beta[J]; m.WlJ = maxZl[J];
        m.c0 = c0; m.nvJ = nv;
    }
}

// One work chunk: R tile, its table entry and a range of items (S tiles).  In CTA-pair mode chunk c
// is (R tile pair t, S tiles [64 jc, 64 jc + 64)) with t = c mod nT; CTA `rank` of the pair takes R
// tile 2t + rank (a tile past the end gets no valid rows) and item e is S tile e.
template <bool kPair>
TJ_DEV void chunk_at(const ScreenArgs& a, unsigned c, unsigned rank, unsigned& rtile, uint4& rt, unsigned& e0,
                     unsigned& e1) {
    if (!kPair) {
        const uint4 ch = a.chunks[c];
        rtile = ch.x;
        rt = a.rtiles[ch.x];
        e0 = ch.y;
        e1 = ch.z;
        return;
    }
    const unsigned t = c % a.nT, jc = c / a.nT;
    e0 = jc * 64u;
    e1 = min(e0 + 64u, a.ntS);
    rtile = 2u * t + rank;
    if (rtile < a.ntR) {
        rt = a.rtiles[rtile];
    } else {
        const uint4 r0 = a.rtiles[2u * t];
        rt = make_uint4(r0.x + (unsigned)kTileR, 0u, r0.z, r0.w);
    }
}

// kFmt: 0 = fp16, 1 = bf16; kSplit: hi/lo operand limbs; kPair: CTA-pair MMA (cta_group::2, no split)
// kTimes: stall accounting (ScreenArgs::role_t) compiled in; the production screens are built without it
template <int kFmt, int kSplit, bool kPair, bool kTimes = false>
__global__ void __launch_bounds__(kScreenThreads, 1)
    screen_tc_kernel(const __grid_constant__ TMaps tm, const ScreenArgs a) {
    using Cfg = typename StageSel<kSplit, kPair>::type;
    constexpr int kStages = Cfg::kStages;
    constexpr unsigned kStageBytes = Cfg::kBytes;
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    uint8_t* smem = (uint8_t*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    ColMetaHot* meta = (ColMetaHot*)(smem + (size_t)kStages * kStageBytes);
    __shared__ long long role_acc[kScreenThreads / 32][6];   // stall accounting per warp (TJ_FLAG_SCREEN_TIMES)
    ScreenCtl<kStages>* ctl = (ScreenCtl<kStages>*)(meta + kMetaSlots);
    const unsigned warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    unsigned long long* status = &a.ctr->status;
    const unsigned rank = kPair ? cluster_ctarank() : 0u;   // 0: the pair's MMA-issuing CTA

    if (threadIdx.x == 0) {
        for (int s = 0; s < kStages; ++s) {
            mbar_init(&ctl->full[s], 1);
            mbar_init(&ctl->empty[s], 1);
        }
        for (int b = 0; b < kAccMax; ++b) {
            mbar_init(&ctl->acc_full[b], 1);
            // pair: the 12 epilogue warps of both CTAs; one SM: the 4 warps of one epilogue group
            mbar_init(&ctl->acc_empty[b], kPair ? 2 * kEpiWarps : 4);
        }
        for (int m = 0; m < kMetaSlots; ++m) {
            mbar_init(&ctl->meta_full[m], 1);
            // pair: the 12 epilogue warps; one SM: the 8 warps of the item's two half-items (4 warps
            // arriving twice where only one half is live)
            mbar_init(&ctl->meta_empty[m], kPair ? kEpiWarps : 8);
        }
        mbar_init(&ctl->drain, 1);
        for (int r = 0; r < kChunkRing; ++r) {
            mbar_init(&ctl->cfull[r], 1);
            mbar_init(&ctl->cempty[r], 1 + kEpiWarps);   // the UMMA issuer and every epilogue warp
        }
        ctl->abort_flag = 0;
        fence_barrier_init();
        for (int c = 0; c < a.ncls; ++c) {
            prefetch_tmap(&tm.a[c]);
            prefetch_tmap(&tm.b[c]);
        }
    }
    if (warp == 1) {
        if (kPair) tmem_alloc_pair(&ctl->tmem_base, 512);
        else tmem_alloc(&ctl->tmem_base, 512);
    }
    tc_fence_before();
    if (kPair) cluster_sync();   // the peer's barriers are initialised before any remote arrival
    else __syncthreads();
    tc_fence_after();
    const unsigned tmem = ctl->tmem_base;
    const unsigned nchunks = kPair ? a.nT * ((a.ntS + 63u) / 64u) : *a.nchunks;
    const int nst = (a.nstages >= 2 && a.nstages <= kStages) ? a.nstages : kStages;
    const unsigned cfirst = kPair ? (blockIdx.x >> 1) : blockIdx.x;
    const unsigned cstride = kPair ? (gridDim.x >> 1) : gridDim.x;
    if (a.cta_t && threadIdx.x == 0) a.cta_t[2 * blockIdx.x] = global_ns();

    if (warp == 0) {
        // ------------------------------------------------------------ TMA producer
        if (lane == 0) {
            unsigned stage = 0, phase = 0;
            unsigned long long n = 0;   // items issued
            bool ok = true;
            const long long t_role = kTimes ? clock64() : 0;
            long long w_stage = 0, w_meta = 0;
            for (unsigned long long qc = 0;; ++qc) {
                unsigned c;
                if (kPair) {   // the two CTAs of a pair walk the same static sequence
                    c = cfirst + (unsigned)qc * cstride;
                    if (c >= nchunks || !ok) break;
                } else {       // first wave by CTA index, then the device queue
                    c = qc == 0 ? blockIdx.x : gridDim.x + (unsigned)atomicAdd(&a.ctr->chunk_next, 1ull);
                    const bool end = !ok || c >= nchunks;
                    if (!publish_chunk(ctl, qc, end ? kNoChunk : c, status, a.wait_ns)) { ok = false; break; }
                    if (end) break;
                }
                unsigned rtile, e0, e1;
                uint4 rt;
                chunk_at<kPair>(a, c, rank, rtile, rt, e0, e1);
                if (a.join_t) atomicMin(&a.join_t[rt.z], global_ns());
                const int rrow = (int)rt.x;
                const unsigned cls = rt.w;
                const int kblocks = a.cls[cls].kblocks, kpad = a.cls[cls].kpad, kbk = a.cls[cls].kbk;
                const unsigned tx = a.cls[cls].tx_bytes;
                const CUtensorMap* mA = &tm.a[cls];
                const CUtensorMap* mB = &tm.b[cls];
                for (unsigned e = e0; e < e1 && ok; ++e) {
                    unsigned J = e, hm = 3u;   // one SM: live 128-row halves of the S tile
                    if (!kPair) {
                        const uint32_t je = a.jlist[e];
                        J = je & kJMask;
                        if (a.half) hm = je >> 30;
                        if (!hm) continue;
                    }
                    const int srow = (int)a.stiles[J].x + (int)(rank * kTileR);   // pair: this CTA's half
                    const unsigned slot = (unsigned)(n % kMetaSlots), mph = (unsigned)((n / kMetaSlots) & 1);
                    const long long t_m = kTimes ? clock64() : 0;
                    if (!mbar_wait(&ctl->meta_empty[slot], mph ^ 1, status, a.wait_ns)) { ok = false; break; }
                    if (kTimes) w_meta += clock64() - t_m;
                    mbar_arrive_expect_tx(&ctl->meta_full[slot], (unsigned)sizeof(ColMetaHot));
                    bulk_load(&meta[slot], (const ColMetaHot*)(a.s_meta + J), (unsigned)sizeof(ColMetaHot),
                              &ctl->meta_full[slot]);
                    for (int kb = 0; kb < kblocks; ++kb) {
                        const long long t_s = kTimes ? clock64() : 0;
                        if (!mbar_wait(&ctl->empty[stage], phase ^ 1, status, a.wait_ns)) { ok = false; break; }
                        if (kTimes) w_stage += clock64() - t_s;
                        if (*(volatile int*)&ctl->abort_flag) { ok = false; break; }
                        uint8_t* sa = smem + (size_t)stage * kStageBytes;
                        if (kPair) {   // both CTAs' copies complete on the MMA CTA's barrier
                            const unsigned fb = mapa_shared(&ctl->full[stage], 0);
                            if (rank == 0) mbar_arrive_expect_tx(&ctl->full[stage], 2 * tx);
                            tma_load_2d_pair(sa, mA, fb, kb * kbk, rrow);
                            tma_load_2d_pair(sa + Cfg::kBhi, mB, fb, kb * kbk, srow);
                        } else {   // A, then each live 128-row half of B (hi, and lo with the split)
                            const unsigned bhalf = 256u * (unsigned)kbk;
                            mbar_arrive_expect_tx(&ctl->full[stage],
                                                  a.cls[cls].tx_a + (unsigned)__popc(hm) * a.cls[cls].tx_h);
                            tma_load_2d(sa, mA, &ctl->full[stage], kb * kbk, rrow);
                            if (kSplit) tma_load_2d(sa + Cfg::kAlo, mA, &ctl->full[stage], kpad + kb * kbk, rrow);
#pragma unroll
                            for (int h = 0; h < 2; ++h) {
                                if (!((hm >> h) & 1u)) continue;
                                tma_load_2d(sa + Cfg::kBhi + h * bhalf, mB, &ctl->full[stage], kb * kbk, srow + h * 128);
                                if (kSplit)
                                    tma_load_2d(sa + Cfg::kBlo + h * bhalf, mB, &ctl->full[stage], kpad + kb * kbk,
                                                srow + h * 128);
                            }
                        }
                        if (++stage == nst) { stage = 0; phase ^= 1; }
                    }
                    ++n;
                }
            }
            if (!ok) ctl->abort_flag = 1;
            if (kTimes) {
                atomicAdd(&a.role_t[kRoleProd], (unsigned long long)(clock64() - t_role));
                atomicAdd(&a.role_t[kRoleProdStage], (unsigned long long)w_stage);
                atomicAdd(&a.role_t[kRoleProdMeta], (unsigned long long)w_meta);
            }
            // drain: the last copy issued into every stage / metadata slot must land before exit.  In
            // the pair the stage barriers live in CTA 0 and count both CTAs' copies: CTA 0 waits for
            // the phases it armed, and CTA 1, which cannot see them, waits for its own stages to be
            // released by the pair's MMA (its `empty` barriers, signalled after the MMA that read
            // the copy); where the MMA stopped early these waits run out after kDrainLimitNs each,
            // long after any copy issued has landed.  The final cluster barrier follows both.
            for (int s = 0; s < nst; ++s) {
                const unsigned ph = ((unsigned)s < stage) ? phase : (phase ^ 1u);
                if (rank == 0) mbar_wait(&ctl->full[s], ph, status, kDrainLimitNs);
                else if (n > 0) mbar_wait(&ctl->empty[s], ph, status, kDrainLimitNs);
            }
            for (int s = 0; s < kMetaSlots; ++s) {
                if (n <= (unsigned long long)s) continue;
                const unsigned long long last = ((n - 1 - s) / kMetaSlots) * kMetaSlots + s;
                mbar_wait(&ctl->meta_full[s], (unsigned)((last / kMetaSlots) & 1), status, kDrainLimitNs);
            }
        }
    } else if (warp == 1) {
        // ------------------------------------------------------------ UMMA issuer (pair: CTA 0 only)
        if (lane == 0 && rank == 0) {
            unsigned stage = 0, phase = 0, acc = 0, acc_phase = 0;
            unsigned long long n_mma = 0;   // items issued
            unsigned ns = 0;                // one SM: half-items issued
            bool ok = true;
            const long long t_role = kTimes ? clock64() : 0;
            long long w_op = 0, w_acc = 0;
            for (unsigned long long qc = 0;; ++qc) {
                unsigned c;
                if (kPair) {
                    c = cfirst + (unsigned)qc * cstride;
                    if (c >= nchunks || !ok) break;
                } else {
                    if (!ok) break;
                    if (!take_chunk(ctl, qc, c, status, a.wait_ns, false)) { ok = false; break; }
                    if (c == kNoChunk) break;
                }
                unsigned rtile, e0, e1;
                uint4 rt;
                chunk_at<kPair>(a, c, 0u, rtile, rt, e0, e1);
                const ScreenClassArgs& ca = a.cls[rt.w];
                const int kblocks = ca.kblocks, ksteps = ca.kbk / 16;
                const uint32_t dh = ca.desc_hi;
                for (unsigned e = e0; e < e1 && ok; ++e) {
                    unsigned hm = 3u;   // one SM: live 128-row halves of the item's S tile
                    if (!kPair && a.half) {
                        hm = a.jlist[e] >> 30;
                        if (!hm) continue;
                    }
                    // one SM: live half h takes the next half-item s = ns, ns + 1, ... (accumulator s mod 4)
                    unsigned bh[2] = {0u, 0u};
                    bool got = true;
                    const long long t_a = kTimes ? clock64() : 0;
                    if (kPair) {
                        got = mbar_wait_cluster(&ctl->acc_empty[acc], acc_phase ^ 1, status, a.wait_ns);
                    } else {
#pragma unroll
                        for (int h = 0; h < 2; ++h) {
                            if (!((hm >> h) & 1u)) continue;
                            bh[h] = (unsigned)(ns & 3);
                            got = got && mbar_wait(&ctl->acc_empty[bh[h]], (unsigned)((ns >> 2) & 1) ^ 1u, status,
                                                   a.wait_ns);
                            ++ns;
                        }
                    }
                    if (!got) { ok = false; break; }
                    if (kTimes) w_acc += clock64() - t_a;
                    tc_fence_after();
                    const unsigned d_tmem = tmem + acc * kTileS;                 // pair: 256 columns
                    const unsigned d0 = tmem + bh[0] * 128u, d1 = tmem + bh[1] * 128u;   // one SM: 2 x 128
                    const unsigned bhalf = 256u * (unsigned)ca.kbk;              // bytes of 128 B rows
                    for (int kb = 0; kb < kblocks; ++kb) {
                        const long long t_o = kTimes ? clock64() : 0;
                        if (!mbar_wait(&ctl->full[stage], phase, status, a.wait_ns)) { ok = false; break; }
                        if (kTimes) w_op += clock64() - t_o;
                        if (*(volatile int*)&ctl->abort_flag) { ok = false; break; }
                        tc_fence_after();
                        const uint8_t* sa = smem + (size_t)stage * kStageBytes;
#pragma unroll
                        for (int k = 0; k < kBK / 16; ++k) {
                            if (k >= ksteps) break;
                            const unsigned accum = (kb | k) != 0 ? 1u : 0u;
                            const uint64_t ad = desc_kmajor(sa, k * 32, dh);
                            if (kPair) {
                                umma_f16_pair(d_tmem, ad, desc_kmajor(sa + Cfg::kBhi, k * 32, dh), a.idesc_pair, accum);
                            } else {
#pragma unroll
                                for (int h = 0; h < 2; ++h) {
                                    if (!((hm >> h) & 1u)) continue;
                                    const unsigned dd = h ? d1 : d0;
                                    const uint64_t bd = desc_kmajor(sa + Cfg::kBhi + h * bhalf, k * 32, dh);
                                    umma_f16(dd, ad, bd, a.idesc, accum);
                                    if (kSplit) {   // z.w ~ hi.hi + hi.lo + lo.hi, one FP32 accumulator
                                        umma_f16(dd, ad, desc_kmajor(sa + Cfg::kBlo + h * bhalf, k * 32, dh), a.idesc,
                                                 1u);
                                        umma_f16(dd, desc_kmajor(sa + Cfg::kAlo, k * 32, dh), bd, a.idesc, 1u);
                                    }
                                }
                            }
                        }
                        if (kPair) umma_commit_pair_mc(&ctl->empty[stage], 0x3);   // frees the stage in both CTAs
                        else umma_commit(&ctl->empty[stage]);
                        if (++stage == nst) { stage = 0; phase ^= 1; }
                    }
                    if (!ok) break;
                    if (kPair) {
                        umma_commit_pair_mc(&ctl->acc_full[acc], 0x3);   // both CTAs' epilogues
                        if (++acc == 2) { acc = 0; acc_phase ^= 1; }
                    } else {
                        if (hm & 1u) umma_commit(&ctl->acc_full[bh[0]]);
                        if (hm & 2u) umma_commit(&ctl->acc_full[bh[1]]);
                    }
                    ++n_mma;
                }
            }
            if (!kPair && n_mma) atomicAdd(&a.ctr->items, n_mma);
            if (!ok) ctl->abort_flag = 1;
            if (kTimes) {
                atomicAdd(&a.role_t[kRoleMma], (unsigned long long)(clock64() - t_role));
                atomicAdd(&a.role_t[kRoleMmaOperand], (unsigned long long)w_op);
                atomicAdd(&a.role_t[kRoleMmaAcc], (unsigned long long)w_acc);
            }
            if (kPair) umma_commit_pair_mc(&ctl->drain, 0x1);
            else umma_commit(&ctl->drain);
            mbar_wait(&ctl->drain, 0, status, kDrainLimitNs);
        }
    } else if (warp >= kEpiFirst) {
        // ------------------------------------------------------------ epilogue
        const unsigned q = warp & 3;                 // TMEM lane quarter of this warp
        const unsigned part = (warp - kEpiFirst) >> 2;   // pair: column third; one SM: epilogue group
        const unsigned row = q * 32 + lane;              // R row within the tile
        // pair: 32-column blocks of the 256-column accumulator, thirds [0, 3), [3, 6), [6, 8);
        // one SM: all four blocks of a 128-column half-item (sub-item s = 2 item + half, taken by
        // group s mod 3, accumulator s mod 4)
        const int cb_begin = kPair ? (int)part * 3 : 0;
        const int cb_end = kPair ? (part == 2 ? kTileS / 32 : (int)part * 3 + 3) : 4;
        WarpAppender app_acc, app_band;
        unsigned acc = 0, acc_phase = 0;
        unsigned long long n_screen_acc = 0, n_rare = 0, n_items = 0;
        unsigned n = 0, ns = 0;   // items, and (one SM) half-items passed: the UMMA issuer's numbering
        bool ok = true;
        // stall accounting in shared memory (lane 0 of each warp), so that it costs no registers
        long long* racc = role_acc[warp];
        if (kTimes && lane == 0) {
            racc[0] = clock64();
            for (int k = 1; k < 6; ++k) racc[k] = 0;
        }
        for (unsigned long long qc = 0;; ++qc) {
            unsigned c;
            if (kPair) {
                c = cfirst + (unsigned)qc * cstride;
                if (c >= nchunks || !ok) break;
            } else {
                if (!ok) break;
                if (!take_chunk(ctl, qc, c, status, a.wait_ns, true)) { ok = false; break; }
                if (c == kNoChunk) break;
            }
            unsigned rtile, e0, e1;
            uint4 rt;
            chunk_at<kPair>(a, c, rank, rtile, rt, e0, e1);
            const ScreenClassArgs& ca = a.cls[rt.w];
            const JoinParams& jp = a.jps[rt.z];   // read through L1 where used
            const unsigned r0 = rt.x;
            const bool rvalid = row < rt.y;
            const unsigned rs = r0 + row;
            const double Ai = rvalid ? ca.r_nrm2[rs] : 0.0;
            // row bounds held as FP32 (exact in FP64, widened where used)
            const float Zi = rvalid ? ca.r_zn[rs] : 0.f;
            const float Ei = rvalid ? ca.r_en[rs] : 0.f;
            const float Zli = rvalid ? ca.r_zl[rs] : 0.f;
            const uint32_t oi = rvalid ? ca.r_emit[rs] : 0u;
            // the row's parts of the per-item thresholds below (FP64; every sum keeps the margins
            // that cover its rounding)
            const double Zd = Zi, Ed = Ei, Zld = Zli;
            const double cabs = jp.cabs;
            const double zg = jp.gmma * Zd, pz = Zd * (1.0 + jp.gmma), gA = jp.gn * Ai;
            const double tp_base = jp.Tp - Ai + 0x1p-50 * (jp.Tp + Ai) + 0x1p-1000;
            const double tm_base = jp.Tm - Ai - 0x1p-50 * (jp.Tm + Ai) - 0x1p-1000;
            for (unsigned e = e0; e < e1 && ok; ++e) {
              unsigned hm = 3u;   // one SM: live 128-row halves of the item's S tile
              if (!kPair && a.half) {
                  hm = a.jlist[e] >> 30;
                  if (!hm) continue;
              }
              // the item's metadata slot is read and released only by the warps whose group takes one
              // of its half-items (consecutive half-items go to different groups)
              const unsigned slot = (unsigned)(n % kMetaSlots), mph = (unsigned)((n / kMetaSlots) & 1);
              const unsigned meta_arrivals = (!kPair && __popc(hm) == 1) ? 2u : 1u;
              for (unsigned h = 0; h < (kPair ? 1u : 2u); ++h) {
                unsigned colbase = 0, b = acc, bph = acc_phase;
                if (!kPair) {   // live half h is half-item ns: group ns mod 3, accumulator ns mod 4
                    if (!((hm >> h) & 1u)) continue;
                    const unsigned sub = ns++;
                    if ((unsigned)(sub % 3) != part) continue;
                    colbase = h * 128u;
                    b = (unsigned)(sub & 3);
                    bph = (unsigned)((sub >> 2) & 1);
                }
                if (kTimes && lane == 0) racc[1] -= clock64();
                if (!__all_sync(0xffffffffu, mbar_wait(&ctl->meta_full[slot], mph, status, a.wait_ns))) {
                    ok = false;
                    break;
                }
                if (kTimes && lane == 0) racc[1] += clock64();
                const ColMetaHot& m = meta[slot];
                const unsigned c0 = m.c0;
                // per-(row, S tile) fast threshold; every error term bounded by tile maxima
                //   v > tau       =>  D > Tp  (certainly out)
                //   v <= tau_in   =>  D <= Tm (certainly in)
                float tau = -INFINITY, tau_in = -INFINITY;
                if (rvalid) {
                    const double WJ = m.WJ, FJ = m.FJ, YJ = m.YJ, BJ = m.BJ, betaJ = m.betaJ, WlJ = m.WlJ;
                    const double RiJ = zg * WJ + cabs + Ed * YJ + Zd * FJ + Zld * WlJ;
                    const double PiJ = pz * WJ + cabs;
                    const double slack = gA + 0x1p-23 * (BJ + 2.0 * PiJ) + betaJ + 2.0 * RiJ;
                    // the 2^-40 / 2^-50 terms exceed the FP64 rounding of these sums even under cancellation
                    tau = f32_up(tp_base + slack * (1.0 + 0x1p-40));
                    tau_in = f32_dn(tm_base - slack * (1.0 + 0x1p-40));
                }
                // the thresholds above need only the metadata: the accumulator is awaited after them
                // (warp-uniform: the TMEM loads below are warp-collective)
                if (kTimes && lane == 0) racc[2] -= clock64();
                if (!__all_sync(0xffffffffu, mbar_wait(&ctl->acc_full[b], bph, status, a.wait_ns))) {
                    ok = false;
                    break;
                }
                if (kTimes && lane == 0) {
                    const long long now = clock64();
                    racc[2] += now;
                    racc[3] -= now;
                }
                tc_fence_after();
                const unsigned tbase = tmem + ((q * 32u) << 16) + (kPair ? b * kTileS : b * 128u);
                if (a.dump && e % a.dump_every == 0 && e / a.dump_every < a.dump_items) {
                    // diagnostics: the raw accumulators of sampled items, in a rolled pass of its own
                    // (kept out of the unrolled test below, whose code must stay in the instruction cache)
                    const size_t slotd = e / a.dump_every;
#pragma unroll 1
                    for (int c8 = cb_begin * 4; c8 < cb_end * 4; ++c8) {   // 8 columns per TMEM load
                        const int col0 = (int)colbase + c8 * 8;
                        uint32_t raw[8];
                        tmem_ld8(tbase + c8 * 8, raw);
                        tmem_ld_wait();
                        float* out = a.dump + (slotd * kTileR + row) * kTileS + col0;
#pragma unroll
                        for (int k = 0; k < 8; ++k) out[k] = __uint_as_float(raw[k]);
                        if (row == 0 && col0 == 0) a.dump_ids[slotd] = make_uint4(rtile, a.jlist[e] & kJMask, 1u, 0u);
                    }
                }
                // phase 1: every 32-column block of this warp's part is read from TMEM and tested; a
                // lane keeps, per block, the mask of its candidates (v <= tau) and of the certified
                // accepts among them (v <= tau_in).  No warp-collective step runs here, and the
                // accumulator is handed back as soon as the last block is in registers.  The block loop
                // stays rolled (one copy of the test in the instruction cache); the per-block masks sit
                // in a small per-thread array indexed by block.
                uint32_t cmk[4] = {0u, 0u, 0u, 0u}, imk[4] = {0u, 0u, 0u, 0u};
#pragma unroll 1
                for (int i = 0; i < 4; ++i) {
                    const int cb = cb_begin + i;
                    if (cb >= cb_end) break;
                    const int col0 = (int)colbase + cb * 32;   // column of the S tile
                    uint32_t raw[32];
                    tmem_ld32(tbase + cb * 32, raw);
                    tmem_ld_wait();
                    if (cb == cb_end - 1) {   // this warp's part read: hand it back
                        tc_fence_before();
                        __syncwarp();
                        if (lane == 0) {
                            if (kPair) mbar_arrive_cluster(mapa_shared(&ctl->acc_empty[b], 0));
                            else mbar_arrive(&ctl->acc_empty[b]);
                        }
                    }
                    uint32_t cm = 0, im = 0;
                    if (kPair) {
                        // dense joins (CTA pair): one test per 8-column group, w = fma(-2, max p, min B~),
                        // a lower bound of every pair's v = fma(-2, p, B~) in the group with the same
                        // magnitude bounds (so the same rounding allowance in tau); four three-input maxes
                        // and one FMA per 8 pairs; only the groups whose value passes tau are examined
                        // pair by pair
                        // (the same test over the whole 32-column block first: one compare and branch
                        // per block while no pair of the block is near the threshold)
                        const float4 gb = *reinterpret_cast<const float4*>(&m.gminB[col0 >> 3]);
                        const float gbv[4] = {gb.x, gb.y, gb.z, gb.w};
                        float pmv[4];
#pragma unroll
                        for (int g = 0; g < 4; ++g) {
                            const uint32_t* r8 = raw + 8 * g;
                            pmv[g] = fmax3(fmax3(fmax3(__uint_as_float(r8[0]), __uint_as_float(r8[1]),
                                                       __uint_as_float(r8[2])),
                                                 __uint_as_float(r8[3]), __uint_as_float(r8[4])),
                                           fmaxf(__uint_as_float(r8[5]), __uint_as_float(r8[6])),
                                           __uint_as_float(r8[7]));
                        }
                        const float pblk = fmaxf(fmax3(pmv[0], pmv[1], pmv[2]), pmv[3]);
                        const float bblk = fminf(fmin3(gbv[0], gbv[1], gbv[2]), gbv[3]);
                        if (fmaf(-2.f, pblk, bblk) <= tau) {
#pragma unroll
                        for (int g = 0; g < 4; ++g) {
                            const float pm = pmv[g];
                            if (fmaf(-2.f, pm, gbv[g]) <= tau) {
#pragma unroll
                                for (int k = 8 * g; k < 8 * g + 8; ++k) {
                                    const float v = fmaf(-2.f, __uint_as_float(raw[k]), m.nrm2f[col0 + k]);
                                    cm |= (v <= tau ? 1u : 0u) << k;
                                    im |= (v <= tau_in ? 1u : 0u) << k;
                                }
                            }
                        }
                        }
                    } else {
                        // v = fma(-2, p, B~) two pairs per packed FMA (rounded once, as fmaf), folded by
                        // three-input mins, one min chain per 8-column group: exact per column, which
                        // matters where the norms vary inside a group (clustered data); a group that
                        // passes tau sets its bits from the same eight values
                        const float4* nb4 = reinterpret_cast<const float4*>(&m.nrm2f[col0]);
#pragma unroll
                        for (int g = 0; g < 4; ++g) {
                            const float4 b0 = nb4[2 * g], b1 = nb4[2 * g + 1];
                            const uint32_t* r8 = raw + 8 * g;
                            float v[8];
                            fma_m2_x2(__uint_as_float(r8[0]), __uint_as_float(r8[1]), b0.x, b0.y, v[0], v[1]);
                            fma_m2_x2(__uint_as_float(r8[2]), __uint_as_float(r8[3]), b0.z, b0.w, v[2], v[3]);
                            fma_m2_x2(__uint_as_float(r8[4]), __uint_as_float(r8[5]), b1.x, b1.y, v[4], v[5]);
                            fma_m2_x2(__uint_as_float(r8[6]), __uint_as_float(r8[7]), b1.z, b1.w, v[6], v[7]);
                            const float vm = fmin3(fmin3(fmin3(v[0], v[1], v[2]), v[3], v[4]), fminf(v[5], v[6]), v[7]);
                            if (vm <= tau) {
#pragma unroll
                                for (int k = 0; k < 8; ++k) {
                                    cm |= (v[k] <= tau ? 1u : 0u) << (8 * g + k);
                                    im |= (v[k] <= tau_in ? 1u : 0u) << (8 * g + k);
                                }
                            }
                        }
                    }
                    if (jp.self_join && cm) {   // keep sorted column > sorted row only
                        const int lim = (int)rs - (int)(c0 + col0);   // columns k <= lim: not above the diagonal
                        if (lim >= 31) cm = 0;
                        else if (lim >= 0) cm &= ~((2u << lim) - 1u);
                    }
                    cmk[i] = cm;
                    imk[i] = im & cm;
                }
                // phase 2: one warp scan for the part's certified accepts and band pairs together
                // (accepts in the low 16 bits, band in the high 16: at most 128 of each per lane), one
                // reservation per list, then each lane writes its pairs' canonical keys (these loops stay
                // rolled: four unrolled copies of each overflow the instruction cache)
                if (kTimes && lane == 0) {
                    const long long now = clock64();
                    racc[3] += now;
                    racc[4] -= now;
                }
                const unsigned na = __popc(imk[0]) + __popc(imk[1]) + __popc(imk[2]) + __popc(imk[3]);
                const unsigned nb = __popc(cmk[0] & ~imk[0]) + __popc(cmk[1] & ~imk[1]) + __popc(cmk[2] & ~imk[2]) +
                                    __popc(cmk[3] & ~imk[3]);
                const unsigned packed = na | (nb << 16);
                if (__any_sync(0xffffffffu, packed != 0)) {
                    unsigned tot;
                    const unsigned pre = warp_excl_scan(packed, tot);
                    const unsigned ta = tot & 0xFFFFu, tb = tot >> 16;
                    n_screen_acc += na;
                    n_rare += nb;
                    // one reservation per list (warp-collective); then the warp writes each list's keys
                    // 32 at a time in the warp's order (lane by lane, block by block, column by column):
                    // slot s finds its lane by a shuffle search over the lanes' prefixes and its column
                    // as the right set bit of that lane's masks, so each store of the warp covers 32
                    // consecutive slots and the loop runs once per 32 keys, however unevenly the lanes'
                    // keys fall
                    if (kTimes && lane == 0) racc[5] -= clock64();
                    unsigned long long pa = 0, pb = 0;
                    if (ta) pa = app_acc.reserve(ta, &a.ctr->acc_reserved, a.acc, a.acc_cap);
                    if (tb) pb = app_band.reserve(tb, &a.ctr->band_reserved, a.band, a.band_cap);
                    if (kTimes && lane == 0) racc[5] += clock64();
                    // sparse parts (no lane with more than kDirectMax pairs): every lane writes its own
                    // pairs, accepts and band in one pass in column order, into the same slots the
                    // cooperative loop below would give them (lane by lane, block by block, column by
                    // column), in at most kDirectMax steps of the warp
                    const unsigned most = __reduce_max_sync(0xffffffffu, na + nb);
                    if (most <= kDirectMax) {
                        uint32_t w0 = cmk[0], w1 = cmk[1], w2 = cmk[2], w3 = cmk[3];
                        unsigned long long sa = pa + (pre & 0xFFFFu), sb = pb + (pre >> 16);
#pragma unroll
                        for (unsigned it = 0; it < kDirectMax; ++it) {
                            if (it >= most) break;   // warp-uniform
                            if (w0 | w1 | w2 | w3) {
                                const int blk = w0 ? 0 : w1 ? 1 : w2 ? 2 : 3;
                                const uint32_t w = w0 ? w0 : w1 ? w1 : w2 ? w2 : w3;
                                const uint32_t bit = w & (0u - w);   // lowest set bit
                                const uint32_t acc_w = blk == 0 ? imk[0] : blk == 1 ? imk[1] : blk == 2 ? imk[2] : imk[3];
                                if (blk == 0) w0 ^= bit;
                                else if (blk == 1) w1 ^= bit;
                                else if (blk == 2) w2 ^= bit;
                                else w3 ^= bit;
                                const int col = (int)colbase + (cb_begin + blk) * 32 + (__ffs(bit) - 1);
                                const uint32_t oj = m.perm[col];
                                const uint64_t key = jp.self_join ? pair_key(jp, oi, oj)
                                                                  : jp.key_off + (uint64_t)oi * (uint64_t)jp.n_cols + oj;
                                if (acc_w & bit) {
                                    if (sa < a.acc_cap) a.acc[sa] = key;
                                    ++sa;
                                } else {
                                    if (sb < a.band_cap) a.band[sb] = key;
                                    ++sb;
                                }
                            }
                        }
                    }
#pragma unroll 1
                    for (int list = 0; list < (most <= kDirectMax ? 0 : 2); ++list) {   // 0: certified accepts, 1: band
                        const unsigned tl = list ? tb : ta;
                        if (!tl) continue;   // warp-uniform
                        const unsigned mypre = list ? (pre >> 16) : (pre & 0xFFFFu);
                        uint32_t mk[4];
#pragma unroll
                        for (int i = 0; i < 4; ++i) mk[i] = list ? (cmk[i] & ~imk[i]) : imk[i];
                        uint64_t* buf = list ? a.band : a.acc;
                        const unsigned long long cap = list ? a.band_cap : a.acc_cap;
                        const unsigned long long first = list ? pb : pa;
                        for (unsigned s0 = 0; s0 < tl; s0 += 32) {
                            const unsigned sidx = s0 + lane;
                            unsigned owner = 0;   // the last lane whose prefix is <= sidx
#pragma unroll
                            for (unsigned step = 16; step > 0; step >>= 1) {
                                const unsigned cand = owner + step;   // <= 31
                                if (__shfl_sync(0xffffffffu, mypre, cand) <= sidx) owner = cand;
                            }
                            unsigned j = sidx - __shfl_sync(0xffffffffu, mypre, owner);
                            const uint32_t w0 = __shfl_sync(0xffffffffu, mk[0], owner);
                            const uint32_t w1 = __shfl_sync(0xffffffffu, mk[1], owner);
                            const uint32_t w2 = __shfl_sync(0xffffffffu, mk[2], owner);
                            const uint32_t w3 = __shfl_sync(0xffffffffu, mk[3], owner);
                            const uint32_t ooi = __shfl_sync(0xffffffffu, oi, owner);
                            if (sidx < tl) {
                                const unsigned c0n = __popc(w0), c1n = __popc(w1), c2n = __popc(w2);
                                int blk;
                                uint32_t wsel;
                                if (j < c0n) { blk = 0; wsel = w0; }
                                else if ((j -= c0n) < c1n) { blk = 1; wsel = w1; }
                                else if ((j -= c1n) < c2n) { blk = 2; wsel = w2; }
                                else { j -= c2n; blk = 3; wsel = w3; }
                                const int col = (int)colbase + (cb_begin + blk) * 32 + nth_set_bit(wsel, j);
                                const uint32_t oj = m.perm[col];
                                const uint64_t key = jp.self_join ? pair_key(jp, ooi, oj)
                                                                  : jp.key_off + (uint64_t)ooi * (uint64_t)jp.n_cols + oj;
                                const unsigned long long pos = first + sidx;
                                if (pos < cap) buf[pos] = key;
                            }
                        }
                    }
                }
                __syncwarp();
                if (kTimes && lane == 0) racc[4] += clock64();
                if (lane == 0) mbar_arrive_cnt(&ctl->meta_empty[slot], meta_arrivals);   // done with the slot
                ++n_items;
                if (kPair && ++acc == 2) { acc = 0; acc_phase ^= 1; }
              }
              ++n;
            }
            if (a.join_t && lane == 0) atomicMax(&a.join_t[a.njoins + rt.z], global_ns());
        }
        if (!ok) ctl->abort_flag = 1;
        app_acc.pad(a.acc, a.acc_cap);
        app_band.pad(a.band, a.band_cap);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            n_screen_acc += __shfl_xor_sync(0xffffffffu, n_screen_acc, o);
            n_rare += __shfl_xor_sync(0xffffffffu, n_rare, o);
        }
        if (lane == 0) {   // the screen's accepts and band pairs are exactly what the appenders wrote
            if (n_screen_acc) {
                atomicAdd(&a.ctr->acc_valid, n_screen_acc);
                atomicAdd(&a.ctr->screen_accept, n_screen_acc);
            }
            if (n_rare) {
                atomicAdd(&a.ctr->band_valid, n_rare);
                atomicAdd(&a.ctr->rare_checks, n_rare);
            }
            if (kPair && warp == kEpiFirst && n_items) atomicAdd(&a.ctr->items, n_items);
            if (kTimes) {
                atomicAdd(&a.role_t[kRoleEpi], (unsigned long long)(clock64() - racc[0]));
                for (int k = 1; k < 6; ++k) atomicAdd(&a.role_t[kRoleEpi + k], (unsigned long long)racc[k]);
            }
        }
    }
    tc_fence_before();
    if (kPair) cluster_sync();   // the pair's last MMA (which read both CTAs' stages) has completed
    else __syncthreads();
    tc_fence_after();
    if (warp == 1) {
        if (kPair) tmem_dealloc_pair(tmem, 512);
        else tmem_dealloc(tmem, 512);
    }
    if (a.cta_t && threadIdx.x == 0) a.cta_t[2 * blockIdx.x + 1] = global_ns();
}

// Screen error of the sampled tile pairs: |d2hat - d2| with d2hat = A + B - 2p from the dumped
// accumulator and d2 the sequential FP64 distance of the original rows, and its ratio to the
// certificate's radius (2R + norm terms).  Non-negative doubles are maximised as their bit patterns.
__global__ void __launch_bounds__(256) screen_error_kernel(const ScreenArgs a, const float* dump, const uint4* ids,
                                                           const void* const* rsrc, const void* const* ssrc,
                                                           unsigned long long* out) {
    const uint4 id = ids[blockIdx.x];
    if (id.z != 1) return;
    const uint4 rt = a.rtiles[id.x];
    const uint4 st = a.stiles[id.y];
    const ScreenClassArgs& ca = a.cls[rt.w];
    const JoinParams jp = a.jps[rt.z];
    const ColMetaF& m = a.s_meta[id.y];
    const float* Rrows = (const float*)rsrc[rt.z];
    const float* Srows = (const float*)ssrc[rt.z];
    double emax = 0.0, rmax = 0.0;
    unsigned long long cnt = 0;
    for (int e = threadIdx.x; e < kTileR * kTileS; e += blockDim.x) {
        const int row = e / kTileS, col = e % kTileS;
        if (row >= (int)rt.y || col >= (int)st.y) continue;
        const unsigned rs = rt.x + row;
        const double p = (double)dump[(size_t)blockIdx.x * kTileR * kTileS + e];
        const double Ai = ca.r_nrm2[rs], Bj = m.nrm2[col];
        const double d2hat = Ai + Bj - 2.0 * p;
        const float* x = Rrows + (size_t)ca.r_emit[rs] * jp.d;
        const float* y = Srows + (size_t)m.perm[col] * jp.d;
        double d2 = 0.0;
        for (int k = 0; k < jp.d; ++k) {
            const double t = __dsub_rn((double)x[k], (double)y[k]);
            d2 = __dadd_rn(d2, __dmul_rn(t, t));
        }
        const double Zi = ca.r_zn[rs], Ei = ca.r_en[rs], Zli = ca.r_zl[rs];
        const double R = jp.gmma * Zi * (double)m.zn[col] + jp.cabs + Ei * (double)m.yn[col] +
                         Zi * (double)m.en[col] + Zli * (double)m.zl[col];
        const double bound = 2.0 * R + jp.gn * (Ai + Bj);
        const double err = fabs(d2hat - d2);
        emax = fmax(emax, err);
        rmax = fmax(rmax, bound > 0 ? err / bound : 0.0);
        ++cnt;
    }
    for (int o = 16; o > 0; o >>= 1) {
        emax = fmax(emax, __shfl_xor_sync(0xffffffffu, emax, o));
        rmax = fmax(rmax, __shfl_xor_sync(0xffffffffu, rmax, o));
        cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicMax(out, (unsigned long long)__double_as_longlong(emax));
        atomicMax(out + 1, (unsigned long long)__double_as_longlong(rmax));
        atomicAdd(out + 2, cnt);
    }
}

// ------------------------------------------------------------------ host side
typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_fn() {
    static EncodeTiledFn fn = nullptr;
    if (!fn) {
        cudaDriverEntryPointQueryResult q;
        void* p = nullptr;
        TJ_CUDA(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q));
        if (!p || q != cudaDriverEntryPointSuccess) fail(-2, "cuTensorMapEncodeTiled not available");
        fn = (EncodeTiledFn)p;
    }
    return fn;
}

}  // namespace

// 2-D tensor map over a row-major [rows, cols] matrix of `esize`-byte elements, box = 128 bytes x box_rows,
// 128-byte swizzle (the UMMA K-major canonical layout).
// 2-D tensor map over a row-major [rows, cols] matrix with boxes of box_rows x (box_bytes / esize)
// elements, swizzled by the box row width (32, 64 or 128 bytes).
void make_tmap_2d(CUtensorMap* m, const void* base, long long rows, long long cols, int esize, int box_rows,
                  CUtensorMapDataType dt, int box_bytes) {
    if (box_bytes != 32 && box_bytes != 64 && box_bytes != 128) fail(-1, "make_tmap_2d: box width");
    const cuuint64_t dims[2] = {(cuuint64_t)cols, (cuuint64_t)rows};
    const cuuint64_t strides[1] = {(cuuint64_t)cols * esize};
    const cuuint32_t box[2] = {(cuuint32_t)(box_bytes / esize), (cuuint32_t)box_rows};
    const cuuint32_t estr[2] = {1, 1};
    const CUtensorMapSwizzle sw = box_bytes == 32 ? CU_TENSOR_MAP_SWIZZLE_32B
                                  : box_bytes == 64 ? CU_TENSOR_MAP_SWIZZLE_64B : CU_TENSOR_MAP_SWIZZLE_128B;
    const CUresult r = encode_fn()(m, dt, 2, const_cast<void*>(base), dims, strides, box, estr,
                                   CU_TENSOR_MAP_INTERLEAVE_NONE, sw,
                                   CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) fail(-2, "cuTensorMapEncodeTiled failed (" + std::to_string((int)r) + ")");
}

void screen_tc(const ScreenInput& g, const EmitBuffers& eb, cudaStream_t st) {
    if (g.ncls < 1 || g.ncls > kMaxClass) fail(-1, "screen_tc: bad class count");
    const int scr = g.R[0]->screen;
    const bool bf = scr == kScreenBF16 || scr == kScreenBF16X3;
    const int split = g.R[0]->split;
    TMaps tm;
    memset(&tm, 0, sizeof(tm));
    ScreenArgs a;
    memset(&a, 0, sizeof(a));
    // CTA-pair screen (cta_group::2): one join, no split, rows of at least 256 elements (MMA-bound)
    // and every tile pair a candidate (checked on the device count: one 4-byte read-back)
    bool pair = g.allow_pair && g.ncls == 1 && g.njoins == 1 && !split && !g.dump && !g.jp0.self_join &&
                g.R[0]->kpad >= 256 && g.tR[0]->ntiles > 0 && g.tS[0]->ntiles > 0;
    if (pair) {
        uint32_t tot = 0;
        TJ_CUDA(cudaMemcpyAsync(&tot, g.cand->dev_counts.p, sizeof(tot), cudaMemcpyDeviceToHost, st));
        TJ_CUDA(cudaStreamSynchronize(st));
        pair = (unsigned long long)tot == (unsigned long long)g.tR[0]->ntiles * (unsigned long long)g.tS[0]->ntiles;
    }
    g.used_pair = pair;
    DBuf<ColMetaF> smeta((size_t)std::max(g.ntS_total, 1), st);
    for (int c = 0; c < g.ncls; ++c) {
        const Side& R = *g.R[c];
        const Side& S = *g.S[c];
        const bool ok = R.screen == scr && S.screen == scr && R.split == split && S.split == split &&
                        (bf || scr == kScreenFP16 || scr == kScreenFP16X3) && R.kpad == S.kpad;
        if (!ok) fail(-1, "screen_tc needs matching bf16 / fp16 operands on both sides of every class");
        const CUtensorMapDataType dt = bf ? CU_TENSOR_MAP_DATA_TYPE_BFLOAT16 : CU_TENSOR_MAP_DATA_TYPE_FLOAT16;
        const long long w = (long long)R.kpad * (split ? 2 : 1);
        int kbk = std::min(R.kpad, kBK);
        if (g.k_block && g.k_block < kbk && R.kpad % g.k_block == 0) kbk = g.k_block;   // tuning knob
        if (kbk != 16 && kbk != 32 && kbk != 64) fail(-1, "screen_tc: operand width");
        make_tmap_2d(&tm.a[c], R.op.p, R.rows_pad, w, 2, kTileR, dt, 2 * kbk);
        make_tmap_2d(&tm.b[c], S.op.p, S.rows_pad, w, 2, kTileR, dt, 2 * kbk);   // 128-row boxes (halves)
        const TileSet& tS = *g.tS[c];
        if (tS.ntiles > 0)
            launch(build_col_meta, tS.ntiles, kTileS, 0, st, tS.row0.p, tS.nvalid.p, S.emit, S.nrm2.p, S.nrm2f.p,
                   S.zn.p, S.en.p, S.yn.p, S.zl.p, tS.maxZ.p, tS.maxE.p, tS.maxY.p, tS.maxB.p, tS.beta.p,
                   tS.maxZl.p, smeta.p + g.sbase[c]);
        a.cls[c].r_emit = R.emit;
        a.cls[c].r_nrm2 = R.nrm2.p;
        a.cls[c].r_zn = R.zn.p;
        a.cls[c].r_en = R.en.p;
        a.cls[c].r_zl = R.zl.p;
        a.cls[c].kblocks = R.kpad / kbk;
        a.cls[c].kpad = R.kpad;
        a.cls[c].kbk = kbk;
        a.cls[c].tx_bytes = (unsigned)(2 * kTileR * kbk * 2);   // CTA pair: this CTA's A rows + B half
        a.cls[c].tx_a = (unsigned)((split ? 2 : 1) * kTileR * kbk * 2);
        a.cls[c].tx_h = (unsigned)((split ? 2 : 1) * 128 * kbk * 2);
        a.cls[c].desc_hi = desc_hi_for_rows(2u * (unsigned)kbk);
    }
    a.chunks = g.cand->chunks.p;
    a.nchunks = g.cand->dev_counts.p + 1;
    a.jlist = g.cand->jlist.p;
    a.rtiles = g.rtiles;
    a.stiles = g.stiles;
    a.s_meta = smeta.p;
    a.jps = g.jps;
    a.ncls = g.ncls;
    a.idesc = make_idesc(1u, bf ? 1u : 0u, kTileR, 128u);   // one SM: 128-column half-items
    a.idesc_pair = make_idesc(1u, bf ? 1u : 0u, 2 * kTileR, kTileS);
    a.ntR = (unsigned)g.tR[0]->ntiles;
    a.ntS = (unsigned)g.tS[0]->ntiles;
    a.nT = (a.ntR + 1) / 2;
    a.acc = eb.acc;
    a.acc_cap = eb.acc_cap;
    a.band = eb.band;
    a.band_cap = eb.band_cap;
    a.ctr = eb.ctr;
    a.dump = g.dump;
    a.dump_ids = g.dump_ids;
    a.dump_every = g.dump_every ? g.dump_every : 1u;
    a.dump_items = g.dump ? g.dump_items : 0u;
    a.wait_ns = pipeline_wait_ns();
    a.join_t = g.join_t;
    a.cta_t = g.cta_t;
    a.role_t = g.role_t;
    a.nstages = g.stages;
    a.half = g.half_packed ? 1 : 0;
    a.njoins = (unsigned)g.njoins;
    TJ_CUDA(cudaMemsetAsync(&eb.ctr->chunk_next, 0, sizeof(unsigned long long), st));
    const int grid = num_sms();
#define TJ_SCREEN_T(F, SP, TM)                                                                                \
    do {                                                                                                      \
        TJ_CUDA(cudaFuncSetAttribute(screen_tc_kernel<F, SP, false, TM>,                                      \
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, (int)screen_smem<SP, false>())); \
        launch(screen_tc_kernel<F, SP, false, TM>, grid, kScreenThreads, screen_smem<SP, false>(), st, tm, a); \
    } while (0)
#define TJ_SCREEN(F, SP)                                      \
    do {                                                      \
        if (a.role_t) TJ_SCREEN_T(F, SP, true);               \
        else TJ_SCREEN_T(F, SP, false);                       \
    } while (0)
    if (pair) {
        auto kern = a.role_t ? (bf ? screen_tc_kernel<1, 0, true, true> : screen_tc_kernel<0, 0, true, true>)
                             : (bf ? screen_tc_kernel<1, 0, true> : screen_tc_kernel<0, 0, true>);
        const size_t smem = screen_smem<0, true>();
        TJ_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        cudaLaunchConfig_t cfg = {};
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = 2;
        attr[0].val.clusterDim.y = 1;
        attr[0].val.clusterDim.z = 1;
        cfg.blockDim = dim3(kScreenThreads);
        cfg.dynamicSmemBytes = smem;
        cfg.stream = st;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        cfg.gridDim = dim3((unsigned)(grid & ~1));
        int nclusters = 0;
        TJ_CUDA(cudaOccupancyMaxActiveClusters(&nclusters, kern, &cfg));
        if (nclusters < 1) fail(-2, "screen_tc: no CTA pair fits on the device");
        cfg.gridDim = dim3((unsigned)(2 * std::min(nclusters, grid / 2)));
        count_launch();
        TJ_CUDA(cudaLaunchKernelEx(&cfg, kern, tm, a));
    } else if (bf && split) TJ_SCREEN(1, 1);
    else if (bf) TJ_SCREEN(1, 0);
    else if (split) TJ_SCREEN(0, 1);
    else TJ_SCREEN(0, 0);
#undef TJ_SCREEN
#undef TJ_SCREEN_T
    if (g.dump && g.dump_items)
        launch(screen_error_kernel, g.dump_items, 256, 0, st, a, (const float*)g.dump, (const uint4*)g.dump_ids,
               g.rsrc, g.ssrc, g.diag_out);
}

}  // namespace tj
