// Exact int14 screen on the tensor cores (tcgen05 kind::i8, sm_100a).
//
// Every int14 coordinate q in [-8192, 8191] is split into two signed int8 limbs
// q = 128 h + l, h = floor((q + 64) / 128) in [-64, 64], l in [-64, 63].  For a tile
// pair the kernel accumulates, exactly in INT32 TMEM accumulators,
//     hh = sum h h',   x = sum (h l' + l h'),   ll = sum l l'
// (|hh|, |ll| <= 4096 d, |x| <= 8192 d: no INT32 overflow for any order) and
// recombines q.q' = 16384 hh + 128 x + ll in INT64, so d2 = |q|^2 + |q'|^2 - 2 q.q'
// and the predicate d2 <= T are exact: there is no band and no refinement.
// This is the reference's limb decomposition and exact recombination
// (src/g9_tc_kernels.py:45-66 limb_dot; NUMERICS_G9_INT14.md:5-18), applied to the
// whole screen instead of a refinement subset.
//
// Fast path: q.q' <= 16384 hh + M with M >= |128 x + ll|.  By Cauchy-Schwarz on the limb vectors,
// |x| <= |h||l'| + |l||h'| and |ll| <= |l||l'|, so per (row i, S tile J)
//     M_iJ = 128 (|h_i| L_J + |l_i| H_J) + |l_i| L_J,   H_J, L_J = tile maxima of |h'|, |l'|
// (FP32 upper bounds of the norms, the sum taken in FP64 and rounded up to an integer), and a pair
// is certainly out when 32768 hh + 2 M_iJ < |q|^2 + |q'|^2 - T.  With
// a_iJ = floor((|q_i|^2 - T - 2 M_iJ) / 2^15) and b_j = floor(|q_j|^2 / 2^15) this is the integer
// test  hh - b_j < a_iJ  (two INT32 ops per pair).  Pairs failing it read x and ll and take the
// exact INT64 test.  (The data-independent bound M = d (128 * 8192 + 4096) is ~3x looser on
// uniform int14 rows and sent ~10x more pairs to the exact test.)
//
// TMEM: hh double-buffered (columns 0..255), x and ll single (256..511).  The hh products of an
// item are committed on their own barrier, and the epilogue's fast path (hh only) runs first; each
// epilogue warp then says whether any of its pairs needs the exact test, and with one k-block per
// item (d <= 128) the UMMA issuer computes x / ll only for items where one does (after issuing the
// next item's hh products), so most items cost one limb product instead of four.  With several
// k-blocks x / ll are computed with hh.
// Warp roles (320 threads): warp 0 TMA producer, warp 1 UMMA issuer, warps 2..9 epilogue
// (warp w reads TMEM lanes 32*(w%4).. and columns 64*((w-2)/4)..).
#include <algorithm>
#include <cstddef>

#include <climits>

#include "tj_emit.cuh"
#include "tj_internal.h"

namespace tj {

namespace {

constexpr int kI8Stages = 3;
constexpr int kI8Epi = 8;
constexpr int kI8Threads = (2 + kI8Epi) * 32;
constexpr int kI8N = 128;                        // S tile rows (UMMA N)
constexpr unsigned kPart = 128u * 128u;          // one 128-row x 128-byte swizzled box (16 KB)
constexpr unsigned kI8Stage = 4 * kPart;         // A_h, A_l, B_h, B_l
constexpr unsigned kColHH0 = 0, kColX = 256, kColLL = 384;

constexpr int kI8Meta = 3;

// Column metadata of one 128-row S tile, loaded with one bulk copy per item.
struct ColMetaI8 {
    int bq[kI8N];           // floor(|q_j|^2 / 2^15); 2^30 for rows beyond the tile's points
    uint32_t perm[kI8N];    // original row id
    long long norm[kI8N];   // exact |q_j|^2
    int gminb[kI8N / 8];    // per 8-column group: min of bq (the group-wise fast test)
    uint32_t c0, nvJ;
    float HJ, LJ;           // >= max |h'|, max |l'| over the tile's rows
};
static_assert(sizeof(ColMetaI8) % 16 == 0, "bulk copies need 16-byte multiples");
static_assert(offsetof(ColMetaI8, gminb) % 16 == 0, "group minima are read four at a time");

struct I8Ctl {
    uint64_t full[kI8Stages];
    uint64_t empty[kI8Stages];
    uint64_t acc_full[2];
    uint64_t hh_empty[2];
    uint64_t xl_empty;
    uint64_t xl_full;      // x and ll of the current item are in TMEM (or were skipped)
    uint64_t xl_dec;       // every epilogue warp has said whether it needs x and ll of the item
    uint64_t meta_full[kI8Meta];
    uint64_t meta_empty[kI8Meta];
    uint64_t drain;
    unsigned tmem_base;
    int abort_flag;
    int need[2];           // item parity: some epilogue warp needs x and ll
};

constexpr size_t kI8Smem = 1024 + (size_t)kI8Stages * kI8Stage + kI8Meta * sizeof(ColMetaI8) + sizeof(I8Ctl);

struct I8Args {
    const uint4* chunks;
    const uint32_t* nchunks;
    const uint32_t* jlist;
    const uint32_t* r_row0;
    const uint32_t* r_nvalid;
    const uint32_t* r_perm;
    const long long* r_norm;   // exact |q|^2
    const float* r_hn;         // >= |h| per row
    const float* r_ln;         // >= |l| per row
    const uint32_t* s_row0;
    const ColMetaI8* s_meta;
    int kblocks;               // kpad / 128
    int kpad;
    unsigned idesc;
    long long T;               // integer threshold
    JoinParams jp;
    uint64_t* acc;
    unsigned long long acc_cap;
    Counters* ctr;
    unsigned long long wait_ns;   // limit of every pipeline wait (drains keep kDrainLimitNs)
};

TJ_DEV int floor_shift15(long long v) { return (int)(v >> 15); }   // arithmetic shift = floor division
// a_iJ = floor(v / 2^15) clamped to [-2^30, 2^31 - 1]: |hh - b_j| < 2^30 for every d the screen takes,
// so the clamp never turns a candidate into a rejection (a huge T makes every real pair a candidate)
TJ_DEV int clamp_shift15(long long v) {
    const long long f = v >> 15;
    return f < -(1ll << 30) ? -(1 << 30) : f > 0x7FFFFFFFll ? 0x7FFFFFFF : (int)f;
}
// columns of a 32-column block at and beyond the tile's valid count carry no point
TJ_DEV uint32_t valid_cols(unsigned nv, unsigned cc) {
    return nv >= cc + 32 ? 0xFFFFFFFFu : nv > cc ? ((1u << (nv - cc)) - 1u) : 0u;
}

// r[k] for a runtime k without local memory (fixed 31-select tree).
TJ_DEV uint32_t pick32(const uint32_t (&r)[32], int k) {
    uint32_t a16[16], a8[8], a4[4], a2[2];
#pragma unroll
    for (int i = 0; i < 16; ++i) a16[i] = (k & 16) ? r[i + 16] : r[i];
#pragma unroll
    for (int i = 0; i < 8; ++i) a8[i] = (k & 8) ? a16[i + 8] : a16[i];
#pragma unroll
    for (int i = 0; i < 4; ++i) a4[i] = (k & 4) ? a8[i + 4] : a8[i];
#pragma unroll
    for (int i = 0; i < 2; ++i) a2[i] = (k & 2) ? a4[i + 2] : a4[i];
    return (k & 1) ? a2[1] : a2[0];
}

__global__ void __launch_bounds__(kI8N) build_col_meta_i8(const uint32_t* row0, const uint32_t* nvalid,
                                                         const uint32_t* perm, const long long* norm,
                                                         const float* maxH, const float* maxL, ColMetaI8* out) {
    const unsigned J = blockIdx.x, t = threadIdx.x;
    const unsigned c0 = row0[J], nv = nvalid[J];
    ColMetaI8& m = out[J];
    const bool ok = t < nv;
    const int bq = ok ? floor_shift15(norm[c0 + t]) : 0x40000000;
    m.bq[t] = bq;
    int gb = bq;   // min over the 8 columns t & ~7 .. (t | 7)
    gb = min(gb, __shfl_xor_sync(0xffffffffu, gb, 1));
    gb = min(gb, __shfl_xor_sync(0xffffffffu, gb, 2));
    gb = min(gb, __shfl_xor_sync(0xffffffffu, gb, 4));
    if ((t & 7) == 0) m.gminb[t >> 3] = gb;
    m.perm[t] = ok ? perm[c0 + t] : 0u;
    m.norm[t] = ok ? norm[c0 + t] : 0ll;
    if (t == 0) { m.c0 = c0; m.nvJ = nv; m.HJ = maxH[J]; m.LJ = maxL[J]; }
}

__global__ void __launch_bounds__(kI8Threads, 1)
    screen_i8_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
                     const I8Args a) {
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    uint8_t* smem = (uint8_t*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    ColMetaI8* meta = (ColMetaI8*)(smem + (size_t)kI8Stages * kI8Stage);
    I8Ctl* ctl = (I8Ctl*)(meta + kI8Meta);
    const unsigned warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    unsigned long long* status = &a.ctr->status;

    if (threadIdx.x == 0) {
        for (int s = 0; s < kI8Stages; ++s) {
            mbar_init(&ctl->full[s], 1);
            mbar_init(&ctl->empty[s], 1);
        }
        for (int b = 0; b < 2; ++b) {
            mbar_init(&ctl->acc_full[b], 1);
            mbar_init(&ctl->hh_empty[b], kI8Epi);
        }
        mbar_init(&ctl->xl_empty, kI8Epi);
        mbar_init(&ctl->xl_full, 1);
        mbar_init(&ctl->xl_dec, kI8Epi);
        ctl->need[0] = ctl->need[1] = 0;
        for (int m = 0; m < kI8Meta; ++m) {
            mbar_init(&ctl->meta_full[m], 1);
            mbar_init(&ctl->meta_empty[m], kI8Epi);
        }
        mbar_init(&ctl->drain, 1);
        ctl->abort_flag = 0;
        fence_barrier_init();
        prefetch_tmap(&tmA);
        prefetch_tmap(&tmB);
    }
    if (warp == 1) tmem_alloc(&ctl->tmem_base, 512);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const unsigned tmem = ctl->tmem_base;
    const unsigned nchunks = *a.nchunks;

    if (warp == 0) {
        if (lane == 0) {
            unsigned stage = 0, phase = 0;
            unsigned long long n = 0;
            bool ok = true;
            for (unsigned c = blockIdx.x; c < nchunks && ok; c += gridDim.x) {
                const uint4 ch = a.chunks[c];
                const int rrow = (int)a.r_row0[ch.x];
                for (unsigned e = ch.y; e < ch.z && ok; ++e, ++n) {
                    const unsigned J = a.jlist[e];
                    const int srow = (int)a.s_row0[J];
                    const unsigned slot = (unsigned)(n % kI8Meta), mph = (unsigned)((n / kI8Meta) & 1);
                    if (!mbar_wait(&ctl->meta_empty[slot], mph ^ 1, status, a.wait_ns)) { ok = false; break; }
                    mbar_arrive_expect_tx(&ctl->meta_full[slot], (unsigned)sizeof(ColMetaI8));
                    bulk_load(&meta[slot], a.s_meta + J, (unsigned)sizeof(ColMetaI8), &ctl->meta_full[slot]);
                    for (int kb = 0; kb < a.kblocks; ++kb) {
                        if (!mbar_wait(&ctl->empty[stage], phase ^ 1, status, a.wait_ns)) { ok = false; break; }
                        if (*(volatile int*)&ctl->abort_flag) { ok = false; break; }
                        uint8_t* st = smem + (size_t)stage * kI8Stage;
                        mbar_arrive_expect_tx(&ctl->full[stage], kI8Stage);
                        tma_load_2d(st, &tmA, &ctl->full[stage], kb * 128, rrow);
                        tma_load_2d(st + kPart, &tmA, &ctl->full[stage], a.kpad + kb * 128, rrow);
                        tma_load_2d(st + 2 * kPart, &tmB, &ctl->full[stage], kb * 128, srow);
                        tma_load_2d(st + 3 * kPart, &tmB, &ctl->full[stage], a.kpad + kb * 128, srow);
                        if (++stage == kI8Stages) { stage = 0; phase ^= 1; }
                    }
                }
            }
            if (!ok) ctl->abort_flag = 1;
            for (int s = 0; s < kI8Stages; ++s) {
                const unsigned ph = ((unsigned)s < stage) ? phase : (phase ^ 1u);
                mbar_wait(&ctl->full[s], ph, status, kDrainLimitNs);
            }
            for (int s = 0; s < kI8Meta; ++s) {
                if (n <= (unsigned long long)s) continue;
                const unsigned long long last = ((n - 1 - s) / kI8Meta) * kI8Meta + s;
                mbar_wait(&ctl->meta_full[s], (unsigned)((last / kI8Meta) & 1), status, kDrainLimitNs);
            }
        }
    } else if (warp == 1) {
        if (lane == 0) {
            unsigned stage = 0, phase = 0;
            unsigned long long n = 0;   // item counter of this CTA
            bool ok = true;
            // One k-block per item (d <= 128): the x / ll products are issued lazily, only when an
            // epilogue warp's fast test leaves a pair for the exact test.  The item's operand stage
            // is held until that decision, which is taken after the next item's hh products are
            // issued, so the tensor pipe keeps working meanwhile.  Several k-blocks: x / ll are
            // issued with hh (their stages cannot all be held).
            const bool lazy = a.kblocks == 1;
            bool pending = false;
            unsigned long long pn = 0;
            unsigned pstage = 0;
            unsigned long long n_xl = 0;   // items that took the low-limb products
            auto resolve = [&](unsigned long long mi, unsigned si) -> bool {
                if (!mbar_wait(&ctl->xl_dec, (unsigned)(mi & 1), status, a.wait_ns)) return false;
                volatile int* need = &ctl->need[mi & 1];
                const int needed = *need;
                *need = 0;   // the item two ahead writes it only after this resolve (acc_full order)
                if (needed) {
                    ++n_xl;
                    tc_fence_after();
                    const uint8_t* st = smem + (size_t)si * kI8Stage;
                    const uint8_t *Ah = st, *Al = st + kPart, *Bh = st + 2 * kPart, *Bl = st + 3 * kPart;
                    const unsigned t_x = tmem + kColX, t_ll = tmem + kColLL;
#pragma unroll
                    for (int k = 0; k < 4; ++k) {
                        umma_i8(t_x, desc_sw128(Ah, k * 32), desc_sw128(Bl, k * 32), a.idesc, k != 0);
                        umma_i8(t_x, desc_sw128(Al, k * 32), desc_sw128(Bh, k * 32), a.idesc, 1u);
                        umma_i8(t_ll, desc_sw128(Al, k * 32), desc_sw128(Bl, k * 32), a.idesc, k != 0);
                    }
                }
                umma_commit(&ctl->xl_full);
                umma_commit(&ctl->empty[si]);
                return true;
            };
            for (unsigned c = blockIdx.x; c < nchunks && ok; c += gridDim.x) {
                const uint4 ch = a.chunks[c];
                for (unsigned e = ch.y; e < ch.z && ok; ++e, ++n) {
                    const unsigned b = (unsigned)(n & 1);
                    const unsigned use = (unsigned)((n >> 1) & 1);   // parity of this buffer's use
                    if (!mbar_wait(&ctl->hh_empty[b], use ^ 1, status, a.wait_ns)) { ok = false; break; }
                    tc_fence_after();
                    const unsigned t_hh = tmem + kColHH0 + b * 128, t_x = tmem + kColX, t_ll = tmem + kColLL;
                    if (lazy) {
                        if (!mbar_wait(&ctl->full[stage], phase, status, a.wait_ns)) { ok = false; break; }
                        if (*(volatile int*)&ctl->abort_flag) { ok = false; break; }
                        tc_fence_after();
                        const uint8_t* st = smem + (size_t)stage * kI8Stage;
#pragma unroll
                        for (int k = 0; k < 4; ++k)
                            umma_i8(t_hh, desc_sw128(st, k * 32), desc_sw128(st + 2 * kPart, k * 32), a.idesc, k != 0);
                        umma_commit(&ctl->acc_full[b]);
                        if (pending && !resolve(pn, pstage)) { ok = false; break; }
                        pending = true;
                        pn = n;
                        pstage = stage;
                        if (++stage == kI8Stages) { stage = 0; phase ^= 1; }
                        continue;
                    }
                    for (int kb = 0; kb < a.kblocks; ++kb) {
                        if (!mbar_wait(&ctl->full[stage], phase, status, a.wait_ns)) { ok = false; break; }
                        if (*(volatile int*)&ctl->abort_flag) { ok = false; break; }
                        tc_fence_after();
                        const uint8_t* st = smem + (size_t)stage * kI8Stage;
                        const uint8_t *Ah = st, *Al = st + kPart, *Bh = st + 2 * kPart, *Bl = st + 3 * kPart;
#pragma unroll
                        for (int k = 0; k < 4; ++k)
                            umma_i8(t_hh, desc_sw128(Ah, k * 32), desc_sw128(Bh, k * 32), a.idesc, (kb | k) != 0);
                        // hh is complete after the last k-block's hh products: release it to the
                        // epilogue now, so its fast path overlaps this item's x / ll products
                        if (kb == a.kblocks - 1) umma_commit(&ctl->acc_full[b]);
                        if (kb == 0) {   // x / ll of the previous item must have been read
                            if (!mbar_wait(&ctl->xl_empty, (unsigned)(n & 1) ^ 1u, status, a.wait_ns)) { ok = false; break; }
                            tc_fence_after();
                        }
#pragma unroll
                        for (int k = 0; k < 4; ++k) {
                            umma_i8(t_x, desc_sw128(Ah, k * 32), desc_sw128(Bl, k * 32), a.idesc, (kb | k) != 0);
                            umma_i8(t_x, desc_sw128(Al, k * 32), desc_sw128(Bh, k * 32), a.idesc, 1u);
                            umma_i8(t_ll, desc_sw128(Al, k * 32), desc_sw128(Bl, k * 32), a.idesc, (kb | k) != 0);
                        }
                        umma_commit(&ctl->empty[stage]);
                        if (++stage == kI8Stages) { stage = 0; phase ^= 1; }
                    }
                    if (!ok) break;
                    umma_commit(&ctl->xl_full);
                }
            }
            if (ok && pending) ok = resolve(pn, pstage);
            if (!lazy) n_xl = n;
            if (n_xl) atomicAdd(&a.ctr->xl_items, n_xl);
            if (!ok) ctl->abort_flag = 1;
            umma_commit(&ctl->drain);
            mbar_wait(&ctl->drain, 0, status, kDrainLimitNs);
        }
    } else {
        const unsigned ew = warp - 2;                 // 0..7
        const unsigned q = warp & 3;                  // TMEM lane quarter
        const unsigned half = ew >> 2;                // column half (0: 0..63, 1: 64..127)
        const unsigned row = q * 32 + lane;
        const JoinParams& jp = a.jp;
        WarpAppender app;
        unsigned long long n = 0, n_acc = 0, n_rare = 0, n_items = 0;
        bool ok = true;
        for (unsigned c = blockIdx.x; c < nchunks && ok; c += gridDim.x) {
            const uint4 ch = a.chunks[c];
            const unsigned I = ch.x;
            const unsigned r0 = a.r_row0[I];
            const bool rvalid = row < a.r_nvalid[I];
            const unsigned rs = r0 + row;
            const long long Ai = rvalid ? a.r_norm[rs] : 0;
            const double hi_n = rvalid ? (double)a.r_hn[rs] : 0.0, li_n = rvalid ? (double)a.r_ln[rs] : 0.0;
            const uint32_t oi = rvalid ? a.r_perm[rs] : 0u;
            for (unsigned e = ch.y; e < ch.z; ++e, ++n) {
                const unsigned b = (unsigned)(n & 1);
                const unsigned slot = (unsigned)(n % kI8Meta), mph = (unsigned)((n / kI8Meta) & 1);
                {   // warp-uniform: the TMEM loads below are warp-collective
                    const bool got = mbar_wait(&ctl->meta_full[slot], mph, status, a.wait_ns) &&
                                     mbar_wait(&ctl->acc_full[b], (unsigned)((n >> 1) & 1), status, a.wait_ns);
                    if (!__all_sync(0xffffffffu, got)) { ok = false; break; }
                }
                tc_fence_after();
                const ColMetaI8& m = meta[slot];
                const unsigned c0 = m.c0;
                // a_iJ with M_iJ >= |128 x + ll| for this row and S tile (every term non-negative;
                // the 2^-40 factor and +2 cover the FP64 rounding of the sum and of the ceil)
                int ai = 0x7FFFFFFF;
                if (rvalid) {
                    const double HJ = m.HJ, LJ = m.LJ;
                    const double Md = (128.0 * (hi_n * LJ + li_n * HJ) + li_n * LJ) * (1.0 + 0x1p-40) + 2.0;
                    const long long M = (long long)ceil(Md);
                    ai = clamp_shift15(Ai - a.T - 2 * M);
                }
                const unsigned lane_off = (q * 32u) << 16;
                const unsigned col0 = half * 64;
                uint32_t cms[2] = {0u, 0u};   // pairs left for the exact test, per 32-column block
                uint32_t hv2[2][32];          // both blocks' hh loads in flight together
                tmem_ld32(tmem + lane_off + kColHH0 + b * 128 + col0, hv2[0]);
                tmem_ld32(tmem + lane_off + kColHH0 + b * 128 + col0 + 32, hv2[1]);
                tmem_ld_wait();
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    const unsigned cc = col0 + h * 32;
                    const uint32_t (&hv)[32] = hv2[h];
                    // fast path, one integer test per 8-column group: hh_j - b_j <= max hh - min b, so
                    // max hh - min b < a_iJ proves every pair of the group out (seven maxes and one
                    // subtract per 8 pairs); only the groups that reach the threshold (in any lane) are
                    // examined pair by pair
                    const int4 gb = *reinterpret_cast<const int4*>(&m.gminb[cc >> 3]);
                    const int gbv[4] = {gb.x, gb.y, gb.z, gb.w};
                    int vx[4];
#pragma unroll
                    for (int g = 0; g < 4; ++g) {
                        const uint32_t* h8 = hv + 8 * g;
                        const int m01 = max((int)h8[0], (int)h8[1]), m23 = max((int)h8[2], (int)h8[3]);
                        const int m45 = max((int)h8[4], (int)h8[5]), m67 = max((int)h8[6], (int)h8[7]);
                        vx[g] = max(max(m01, m23), max(m45, m67)) - gbv[g];
                    }
                    const unsigned gmask = (vx[0] >= ai ? 1u : 0u) | (vx[1] >= ai ? 2u : 0u) |
                                           (vx[2] >= ai ? 4u : 0u) | (vx[3] >= ai ? 8u : 0u);
                    const unsigned gunion = __reduce_or_sync(0xffffffffu, gmask);
                    if (!gunion) continue;
                    uint32_t cmask = 0;
#pragma unroll
                    for (int g = 0; g < 4; ++g) {
                        if (!(gunion & (1u << g))) continue;
                        if (gmask & (1u << g)) {
#pragma unroll
                            for (int k = 8 * g; k < 8 * g + 8; ++k)
                                cmask |= ((int)hv[k] - m.bq[cc + k] >= ai ? 1u : 0u) << k;
                        }
                    }
                    cmask &= valid_cols(m.nvJ, cc);
                    if (jp.self_join && cmask) {   // keep sorted column > sorted row only
                        const int lim = (int)rs - (int)(c0 + cc);
                        if (lim >= 31) cmask = 0;
                        else if (lim >= 0) cmask &= ~((2u << lim) - 1u);
                    }
                    cms[h] = cmask;
                }
                // tell the MMA issuer whether this item's x / ll products are needed at all (it skips
                // them when no warp needs them), then wait for them, or for the skip, in every warp:
                // each epilogue warp observes every phase of xl_full, so the parity names this item
                const bool any = __any_sync(0xffffffffu, (cms[0] | cms[1]) != 0);
                if (lane == 0) {
                    if (any) atomicOr(&ctl->need[n & 1], 1);
                    mbar_arrive(&ctl->xl_dec);
                }
                {
                    const bool xl_ok = mbar_wait(&ctl->xl_full, (unsigned)(n & 1), status, a.wait_ns);
                    if (!__all_sync(0xffffffffu, xl_ok)) { ok = false; break; }   // warp-uniform exit
                }
                tc_fence_after();
#pragma unroll 1
                for (int h = 0; h < 2 && any; ++h) {
                    const uint32_t cmask = cms[h];
                    if (!__any_sync(0xffffffffu, cmask != 0)) continue;
                    const unsigned cc = col0 + h * 32;
                    uint32_t hv[32], xv[32], lv[32];
                    tmem_ld32(tmem + lane_off + kColHH0 + b * 128 + cc, hv);
                    tmem_ld32(tmem + lane_off + kColX + cc, xv);
                    tmem_ld32(tmem + lane_off + kColLL + cc, lv);
                    tmem_ld_wait();
                    uint32_t amask = 0, mk = cmask;
                    while (mk) {   // exact INT64 test, one copy of the code
                        const int k = __ffs(mk) - 1;
                        mk &= mk - 1;
                        ++n_rare;
                        const long long dot = (long long)(int)pick32(hv, k) * 16384ll +
                                              (long long)(int)pick32(xv, k) * 128ll + (long long)(int)pick32(lv, k);
                        const long long d2 = Ai + m.norm[cc + k] - 2 * dot;
                        if (d2 <= a.T) amask |= 1u << k;
                    }
                    unsigned ta;
                    const unsigned pa = warp_excl_scan(__popc(amask), ta);
                    if (ta) {
                        unsigned long long pos = app.reserve(ta, &a.ctr->acc_reserved, a.acc, a.acc_cap) + pa;
                        uint32_t mk = amask;
                        while (mk) {
                            const int k = __ffs(mk) - 1;
                            mk &= mk - 1;
                            if (pos < a.acc_cap) a.acc[pos] = pair_key(jp, oi, m.perm[cc + k]);
                            ++pos;
                        }
                        n_acc += __popc(amask);
                    }
                }
                if (!ok) break;
                // this item's hh buffer, the shared x / ll and the metadata slot are free again
                tc_fence_before();
                __syncwarp();
                if (lane == 0) {
                    mbar_arrive(&ctl->hh_empty[b]);
                    mbar_arrive(&ctl->xl_empty);
                    mbar_arrive(&ctl->meta_empty[slot]);
                }
                ++n_items;
            }
        }
        if (!ok) ctl->abort_flag = 1;
        app.pad(a.acc, a.acc_cap);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            n_acc += __shfl_xor_sync(0xffffffffu, n_acc, o);
            n_rare += __shfl_xor_sync(0xffffffffu, n_rare, o);
        }
        if (lane == 0) {
            if (app.valid) atomicAdd(&a.ctr->acc_valid, app.valid);
            if (n_acc) atomicAdd(&a.ctr->screen_accept, n_acc);
            if (n_rare) atomicAdd(&a.ctr->rare_checks, n_rare);
            if (ew == 0 && n_items) atomicAdd(&a.ctr->items, n_items);
        }
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (warp == 1) tmem_dealloc(tmem, 512);
}

// ------------------------------------------------------------------ high-limb screen
// One tensor-core product per pair: hh = sum h h' (exact INT32), and the rest of q.q' bounded,
// |128 x + ll| <= M_iJ (Cauchy-Schwarz on the limb vectors, as above).  Every pair whose interval
//     [A_i + B_j - 32768 hh - 2 M_iJ,  A_i + B_j - 32768 hh + 2 M_iJ]
// lies above T is out (the group fast test, then the same integer test per pair), one that lies at
// or below T is in (exact INT64 test per candidate), and the rest go to the band buffer, where the
// integer refinement decides them from the int16 rows.  Only the h limbs are loaded, and the R
// tile's limbs stay resident in shared memory for all items of a chunk (only S tiles stream), so an
// item costs 16 KB of L2 traffic and kpad / 32 MMAs.
// Warp roles (512 threads): warp 0 TMA producer, warp 1 TMEM allocator + UMMA issuer, warps 2-3
// idle, warps 4..15 epilogue in three groups of four that take alternate items (warp w reads TMEM
// lanes 32 (w % 4).., all 128 columns in two passes of 64), so three warps per SM sub-partition
// overlap their items' latency.
constexpr int kHHMaxKb = 2;                       // resident R k-blocks at most (kpad <= 256)
constexpr int kHHAcc = 4;                         // TMEM accumulators of 128 columns
constexpr int kHHEpi = 12;                        // three groups of four warps, taking alternate items
constexpr int kHHGroups = kHHEpi / 4;
constexpr int kHHEpiFirst = 4;
constexpr int kHHThreads = (kHHEpiFirst + kHHEpi) * 32;

// Shared-memory plan per resident R k-block count: the double-buffered R tile, then as many 16 KB
// S k-block stages as fit (the MMA waits on S tiles that come from HBM: 6 -> 8 stages took the
// 2M-row int14 screen from 561 to 540 ms), and per-item column metadata for every staged item plus
// the four held in TMEM accumulators.
template <int kMaxKb> struct HHCfg {
    static constexpr int kStages = kMaxKb == 1 ? 10 : 8;
    static constexpr int kMeta = kStages + kHHAcc;
    static constexpr unsigned kABytes = kMaxKb * kPart;   // one resident R tile
};

template <int kStages, int kMeta> struct HHCtl {
    uint64_t a_full[2];
    uint64_t a_empty[2];
    uint64_t full[kStages];
    uint64_t empty[kStages];
    uint64_t acc_full[kHHAcc];
    uint64_t acc_empty[kHHAcc];
    uint64_t meta_full[kMeta];
    uint64_t meta_empty[kMeta];
    uint64_t drain;
    unsigned tmem_base;
    int abort_flag;
};

template <int kMaxKb> constexpr size_t hh_smem() {
    using C = HHCfg<kMaxKb>;
    return 1024 + 2 * (size_t)C::kABytes + (size_t)C::kStages * kPart + C::kMeta * sizeof(ColMetaI8) +
           sizeof(HHCtl<C::kStages, C::kMeta>);
}
static_assert(hh_smem<1>() <= 232448 && hh_smem<2>() <= 232448, "227 KB of shared memory per CTA at most");

struct HHArgs {
    I8Args b;                  // tile tables, row data, threshold, output (as the four-product screen)
    uint64_t* band;
    unsigned long long band_cap;
};

template <int kMaxKb>
__global__ void __launch_bounds__(kHHThreads, 1)
    screen_i8_hh_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
                        const HHArgs ha) {
    constexpr int kHHStages = HHCfg<kMaxKb>::kStages;
    constexpr int kHHMeta = HHCfg<kMaxKb>::kMeta;
    constexpr unsigned kHHABytes = HHCfg<kMaxKb>::kABytes;
    using HHCtl = tj::HHCtl<kHHStages, kHHMeta>;
    const I8Args& a = ha.b;
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    uint8_t* smem = (uint8_t*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    uint8_t* abuf = smem;                                       // 2 x kHHABytes
    uint8_t* bbuf = smem + 2 * (size_t)kHHABytes;               // kHHStages x kPart
    ColMetaI8* meta = (ColMetaI8*)(bbuf + (size_t)kHHStages * kPart);
    HHCtl* ctl = (HHCtl*)(meta + kHHMeta);
    const unsigned warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    unsigned long long* status = &a.ctr->status;

    if (threadIdx.x == 0) {
        for (int i = 0; i < 2; ++i) {
            mbar_init(&ctl->a_full[i], 1);
            mbar_init(&ctl->a_empty[i], 1);
        }
        for (int s = 0; s < kHHStages; ++s) {
            mbar_init(&ctl->full[s], 1);
            mbar_init(&ctl->empty[s], 1);
        }
        for (int b = 0; b < kHHAcc; ++b) {
            mbar_init(&ctl->acc_full[b], 1);
            mbar_init(&ctl->acc_empty[b], 4);   // the four warps of the item's epilogue group
        }
        for (int m = 0; m < kHHMeta; ++m) {
            mbar_init(&ctl->meta_full[m], 1);
            mbar_init(&ctl->meta_empty[m], 4);
        }
        mbar_init(&ctl->drain, 1);
        ctl->abort_flag = 0;
        fence_barrier_init();
        prefetch_tmap(&tmA);
        prefetch_tmap(&tmB);
    }
    if (warp == 1) tmem_alloc(&ctl->tmem_base, 512);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const unsigned tmem = ctl->tmem_base;
    const unsigned nchunks = *a.nchunks;
    const int kblocks = a.kblocks;

    if (warp == 0) {
        // ------------------------------------------------------------ TMA producer
        if (lane == 0) {
            unsigned stage = 0, phase = 0;
            unsigned long long n = 0, nc = 0;   // items, chunks issued
            bool ok = true;
            for (unsigned c = blockIdx.x; c < nchunks && ok; c += gridDim.x, ++nc) {
                const uint4 ch = a.chunks[c];
                const int rrow = (int)a.r_row0[ch.x];
                const unsigned ab = (unsigned)(nc & 1);
                if (!mbar_wait(&ctl->a_empty[ab], (unsigned)((nc >> 1) & 1) ^ 1u, status, a.wait_ns)) { ok = false; break; }
                mbar_arrive_expect_tx(&ctl->a_full[ab], (unsigned)kblocks * kPart);
                for (int kb = 0; kb < kblocks; ++kb)
                    tma_load_2d(abuf + ab * kHHABytes + kb * kPart, &tmA, &ctl->a_full[ab], kb * 128, rrow);
                for (unsigned e = ch.y; e < ch.z && ok; ++e, ++n) {
                    const unsigned J = a.jlist[e];
                    const int srow = (int)a.s_row0[J];
                    const unsigned slot = (unsigned)(n % kHHMeta), mph = (unsigned)((n / kHHMeta) & 1);
                    if (!mbar_wait(&ctl->meta_empty[slot], mph ^ 1, status, a.wait_ns)) { ok = false; break; }
                    mbar_arrive_expect_tx(&ctl->meta_full[slot], (unsigned)sizeof(ColMetaI8));
                    bulk_load(&meta[slot], a.s_meta + J, (unsigned)sizeof(ColMetaI8), &ctl->meta_full[slot]);
                    for (int kb = 0; kb < kblocks; ++kb) {
                        if (!mbar_wait(&ctl->empty[stage], phase ^ 1, status, a.wait_ns)) { ok = false; break; }
                        if (*(volatile int*)&ctl->abort_flag) { ok = false; break; }
                        mbar_arrive_expect_tx(&ctl->full[stage], kPart);
                        tma_load_2d(bbuf + (size_t)stage * kPart, &tmB, &ctl->full[stage], kb * 128, srow);
                        if (++stage == kHHStages) { stage = 0; phase ^= 1; }
                    }
                }
            }
            if (!ok) ctl->abort_flag = 1;
            // drain: the last copy issued into every buffer lands before exit
            for (int s = 0; s < kHHStages; ++s) {
                const unsigned ph = ((unsigned)s < stage) ? phase : (phase ^ 1u);
                mbar_wait(&ctl->full[s], ph, status, kDrainLimitNs);
            }
            for (unsigned ab = 0; ab < 2; ++ab) {
                if (nc <= ab) continue;
                const unsigned long long last = ((nc - 1 - ab) / 2) * 2 + ab;
                mbar_wait(&ctl->a_full[ab], (unsigned)((last >> 1) & 1), status, kDrainLimitNs);
            }
            for (int s = 0; s < kHHMeta; ++s) {
                if (n <= (unsigned long long)s) continue;
                const unsigned long long last = ((n - 1 - s) / kHHMeta) * kHHMeta + s;
                mbar_wait(&ctl->meta_full[s], (unsigned)((last / kHHMeta) & 1), status, kDrainLimitNs);
            }
        }
    } else if (warp == 1) {
        // ------------------------------------------------------------ UMMA issuer
        if (lane == 0) {
            unsigned stage = 0, phase = 0;
            unsigned long long n = 0, nc = 0;
            bool ok = true;
            for (unsigned c = blockIdx.x; c < nchunks && ok; c += gridDim.x, ++nc) {
                const uint4 ch = a.chunks[c];
                const unsigned ab = (unsigned)(nc & 1);
                if (!mbar_wait(&ctl->a_full[ab], (unsigned)((nc >> 1) & 1), status, a.wait_ns)) { ok = false; break; }
                tc_fence_after();
                const uint8_t* A = abuf + ab * kHHABytes;
                for (unsigned e = ch.y; e < ch.z && ok; ++e, ++n) {
                    const unsigned b = (unsigned)(n & (kHHAcc - 1));
                    if (!mbar_wait(&ctl->acc_empty[b], (unsigned)((n / kHHAcc) & 1) ^ 1u, status, a.wait_ns)) { ok = false; break; }
                    tc_fence_after();
                    const unsigned d_tmem = tmem + b * 128u;
                    for (int kb = 0; kb < kblocks; ++kb) {
                        if (!mbar_wait(&ctl->full[stage], phase, status, a.wait_ns)) { ok = false; break; }
                        if (*(volatile int*)&ctl->abort_flag) { ok = false; break; }
                        tc_fence_after();
                        const uint8_t* B = bbuf + (size_t)stage * kPart;
#pragma unroll
                        for (int k = 0; k < 4; ++k)
                            umma_i8(d_tmem, desc_sw128(A + kb * kPart, k * 32), desc_sw128(B, k * 32), a.idesc,
                                    (kb | k) != 0);
                        umma_commit(&ctl->empty[stage]);
                        if (++stage == kHHStages) { stage = 0; phase ^= 1; }
                    }
                    if (!ok) break;
                    umma_commit(&ctl->acc_full[b]);
                }
                umma_commit(&ctl->a_empty[ab]);   // the R tile is free once this chunk's MMAs complete
            }
            if (n) atomicAdd(&a.ctr->items, n);
            if (!ok) ctl->abort_flag = 1;
            umma_commit(&ctl->drain);
            mbar_wait(&ctl->drain, 0, status, kDrainLimitNs);
        }
    } else if (warp >= kHHEpiFirst) {
        // ------------------------------------------------------------ epilogue
        const unsigned group = (warp - kHHEpiFirst) >> 2;   // item n goes to group n mod 3
        const unsigned q = warp & 3;                   // TMEM lane quarter
        const unsigned row = q * 32 + lane;
        const unsigned lane_off = (q * 32u) << 16;
        const JoinParams& jp = a.jp;
        WarpAppender app_acc, app_band;
        unsigned long long n = 0, n_acc = 0, n_rare = 0;
        bool ok = true;
        for (unsigned c = blockIdx.x; c < nchunks && ok; c += gridDim.x) {
            const uint4 ch = a.chunks[c];
            const unsigned I = ch.x;
            const unsigned r0 = a.r_row0[I];
            const bool rvalid = row < a.r_nvalid[I];
            const unsigned rs = r0 + row;
            const long long Ai = rvalid ? a.r_norm[rs] : 0;
            const double hi_n = rvalid ? (double)a.r_hn[rs] : 0.0, li_n = rvalid ? (double)a.r_ln[rs] : 0.0;
            const uint32_t oi = rvalid ? a.r_perm[rs] : 0u;
            for (unsigned e = ch.y; e < ch.z; ++e, ++n) {
                if ((unsigned)(n % kHHGroups) != group) continue;
                const unsigned b = (unsigned)(n & (kHHAcc - 1));
                const unsigned slot = (unsigned)(n % kHHMeta), mph = (unsigned)((n / kHHMeta) & 1);
                if (!__all_sync(0xffffffffu, mbar_wait(&ctl->meta_full[slot], mph, status, a.wait_ns))) {
                    ok = false;
                    break;
                }
                const ColMetaI8& m = meta[slot];
                const unsigned c0 = m.c0;
                // M_iJ >= |128 x + ll| for this row and S tile (every term non-negative; the 2^-40 factor
                // and +2 cover the FP64 rounding of the sum and of the ceil); a_iJ as in the header.
                // Only the metadata is needed: the accumulator is awaited after this.
                int ai = 0x7FFFFFFF;
                long long M = 0;
                if (rvalid) {
                    const double HJ = m.HJ, LJ = m.LJ;
                    const double Md = (128.0 * (hi_n * LJ + li_n * HJ) + li_n * LJ) * (1.0 + 0x1p-40) + 2.0;
                    M = (long long)ceil(Md);
                    ai = clamp_shift15(Ai - a.T - 2 * M);
                }
                // warp-uniform: the TMEM loads below are warp-collective
                if (!__all_sync(0xffffffffu, mbar_wait(&ctl->acc_full[b], (unsigned)((n / kHHAcc) & 1), status,
                                                       a.wait_ns))) {
                    ok = false;
                    break;
                }
                tc_fence_after();
                uint32_t hv2[2][32];
                tmem_ld32(tmem + lane_off + b * 128, hv2[0]);
                tmem_ld32(tmem + lane_off + b * 128 + 32, hv2[1]);
                tmem_ld_wait();
                // the warp's 128 columns in two passes of 64 (the second pass's loads hand the
                // accumulator back once they are in registers)
#pragma unroll 1
                for (int pass = 0; pass < 2; ++pass) {
                if (pass == 1) {
                    tmem_ld32(tmem + lane_off + b * 128 + 64, hv2[0]);
                    tmem_ld32(tmem + lane_off + b * 128 + 96, hv2[1]);
                    tmem_ld_wait();
                    tc_fence_before();
                    __syncwarp();
                    if (lane == 0) mbar_arrive(&ctl->acc_empty[b]);   // the accumulator is in registers
                }
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    const unsigned cc = pass * 64 + h * 32;
                    const uint32_t (&hv)[32] = hv2[h];
                    // group fast test: hh_j - b_j <= max hh - min b over 8 columns, so
                    // max hh - min b < a_iJ proves the whole group out.  The rows of every S tile are in
                    // order of their norms (index build), so the group's min b is close to each b_j: on
                    // uniform int14 rows about 4 % of the warp's 32-column blocks have a lane whose group
                    // passes (22 % in Morton order, where a per-pair subtract was the cheaper test).
                    const int4 gb = *reinterpret_cast<const int4*>(&m.gminb[cc >> 3]);
                    const int gbv[4] = {gb.x, gb.y, gb.z, gb.w};
                    unsigned gmask = 0;
#pragma unroll
                    for (int g = 0; g < 4; ++g) {
                        const uint32_t* h8 = hv + 8 * g;
                        const int a3 = __vimax3_s32((int)h8[0], (int)h8[1], (int)h8[2]);
                        const int b3 = __vimax3_s32((int)h8[3], (int)h8[4], (int)h8[5]);
                        const int gm = __vimax3_s32(a3, b3, max((int)h8[6], (int)h8[7]));
                        gmask |= (gm - gbv[g] >= ai ? 1u : 0u) << g;
                    }
                    if (!__any_sync(0xffffffffu, gmask != 0)) continue;
                    uint32_t cmask = 0;
                    if (gmask) {   // b_j read again (volatile): nothing of the group test stays live
                        const volatile int* bqv = &m.bq[cc];
#pragma unroll
                        for (int g = 0; g < 4; ++g) {
                            if (!(gmask & (1u << g))) continue;
#pragma unroll
                            for (int k = 8 * g; k < 8 * g + 8; ++k)
                                cmask |= ((int)hv[k] - bqv[k] >= ai ? 1u : 0u) << k;
                        }
                    }
                    cmask &= valid_cols(m.nvJ, cc);
                    if (jp.self_join && cmask) {   // keep sorted column > sorted row only
                        const int lim = (int)rs - (int)(c0 + cc);
                        if (lim >= 31) cmask = 0;
                        else if (lim >= 0) cmask &= ~((2u << lim) - 1u);
                    }
                    if (!__any_sync(0xffffffffu, cmask != 0)) continue;
                    // candidates: exact INT64 interval test, in / out / band
                    uint32_t amask = 0, bmask = 0, mk = cmask;
                    while (mk) {
                        const int k = __ffs(mk) - 1;
                        mk &= mk - 1;
                        ++n_rare;
                        const long long mid = Ai + m.norm[cc + k] - 32768ll * (long long)(int)pick32(hv, k);
                        if (mid + 2 * M <= a.T) amask |= 1u << k;
                        else if (mid - 2 * M <= a.T) bmask |= 1u << k;
                    }
                    unsigned ta = 0, tb = 0, pa = 0, pb = 0;
                    if (__any_sync(0xffffffffu, amask != 0)) pa = warp_excl_scan(__popc(amask), ta);
                    if (__any_sync(0xffffffffu, bmask != 0)) pb = warp_excl_scan(__popc(bmask), tb);
                    if (ta) {
                        unsigned long long pos = app_acc.reserve(ta, &a.ctr->acc_reserved, a.acc, a.acc_cap) + pa;
                        uint32_t w = amask;
                        while (w) {
                            const int k = __ffs(w) - 1;
                            w &= w - 1;
                            if (pos < a.acc_cap) a.acc[pos] = pair_key(jp, oi, m.perm[cc + k]);
                            ++pos;
                        }
                        n_acc += __popc(amask);
                    }
                    if (tb) {
                        unsigned long long pos = app_band.reserve(tb, &a.ctr->band_reserved, ha.band, ha.band_cap) + pb;
                        uint32_t w = bmask;
                        while (w) {
                            const int k = __ffs(w) - 1;
                            w &= w - 1;
                            if (pos < ha.band_cap) ha.band[pos] = pair_key(jp, oi, m.perm[cc + k]);
                            ++pos;
                        }
                    }
                }
                }
                __syncwarp();
                if (lane == 0) mbar_arrive(&ctl->meta_empty[slot]);
            }
        }
        if (!ok) ctl->abort_flag = 1;
        app_acc.pad(a.acc, a.acc_cap);
        app_band.pad(ha.band, ha.band_cap);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            n_acc += __shfl_xor_sync(0xffffffffu, n_acc, o);
            n_rare += __shfl_xor_sync(0xffffffffu, n_rare, o);
        }
        if (lane == 0) {
            if (app_acc.valid) atomicAdd(&a.ctr->acc_valid, app_acc.valid);
            if (app_band.valid) atomicAdd(&a.ctr->band_valid, app_band.valid);
            if (n_acc) atomicAdd(&a.ctr->screen_accept, n_acc);
            if (n_rare) atomicAdd(&a.ctr->rare_checks, n_rare);
        }
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (warp == 1) tmem_dealloc(tmem, 512);
}

}  // namespace

void make_tmap_2d(CUtensorMap* m, const void* base, long long rows, long long cols, int esize, int box_rows,
                  CUtensorMapDataType dt, int box_bytes);

void screen_i8(const ScreenInput& g, const EmitBuffers& eb, cudaStream_t st) {
    if (g.ncls != 1 || g.njoins != 1) fail(-7, "the int8-limb screen runs one join at a time");
    const Side& R = *g.R[0];
    const Side& S = *g.S[0];
    if (R.screen != kScreenInt8Limb || S.screen != kScreenInt8Limb) fail(-1, "screen_i8 needs int8-limb sides");
    CUtensorMap tmA, tmB;
    make_tmap_2d(&tmA, R.op8.p, R.rows_pad, 2 * (long long)R.kpad, 1, 128, CU_TENSOR_MAP_DATA_TYPE_UINT8, 128);
    make_tmap_2d(&tmB, S.op8.p, S.rows_pad, 2 * (long long)S.kpad, 1, kI8N, CU_TENSOR_MAP_DATA_TYPE_UINT8, 128);
    I8Args a;
    a.chunks = g.cand->chunks.p;
    a.nchunks = g.cand->dev_counts.p + 1;
    a.jlist = g.cand->jlist.p;
    a.r_row0 = g.tR[0]->row0.p;
    a.r_nvalid = g.tR[0]->nvalid.p;
    a.r_perm = R.emit;
    a.r_norm = R.inorm.p;
    a.r_hn = R.zn.p;   // the int8-limb preparation stores |h| and |l| upper bounds in zn / zl
    a.r_ln = R.zl.p;
    const TileSet& tS = *g.tS[0];
    DBuf<ColMetaI8> smeta((size_t)std::max(tS.ntiles, 1), st);
    if (tS.ntiles > 0)
        launch(build_col_meta_i8, tS.ntiles, kI8N, 0, st, tS.row0.p, tS.nvalid.p, S.emit, S.inorm.p, tS.maxZ.p,
               tS.maxZl.p, smeta.p);
    a.s_row0 = tS.row0.p;
    a.s_meta = smeta.p;
    a.kblocks = R.kpad / 128;
    a.kpad = R.kpad;
    a.idesc = make_idesc(2u, 1u, 128, kI8N);
    a.T = g.T_int;
    a.jp = g.jp0;
    a.acc = eb.acc;
    a.acc_cap = eb.acc_cap;
    a.ctr = eb.ctr;
    a.wait_ns = pipeline_wait_ns();
    if (i8_high_limb_screen(g)) {
        HHArgs ha;
        ha.b = a;
        ha.band = eb.band;
        ha.band_cap = eb.band_cap;
        if (a.kblocks == 1) {
            TJ_CUDA(cudaFuncSetAttribute(screen_i8_hh_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)hh_smem<1>()));
            launch(screen_i8_hh_kernel<1>, num_sms(), kHHThreads, hh_smem<1>(), st, tmA, tmB, ha);
        } else {
            TJ_CUDA(cudaFuncSetAttribute(screen_i8_hh_kernel<2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)hh_smem<2>()));
            launch(screen_i8_hh_kernel<2>, num_sms(), kHHThreads, hh_smem<2>(), st, tmA, tmB, ha);
        }
        return;
    }
    TJ_CUDA(cudaFuncSetAttribute(screen_i8_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kI8Smem));
    launch(screen_i8_kernel, num_sms(), kI8Threads, kI8Smem, st, tmA, tmB, a);
}

bool i8_high_limb_screen(const ScreenInput& g) {
    return !g.i8_four_products && g.R[0]->kpad <= kHHMaxKb * 128;
}

}  // namespace tj
