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
// Fast path (every pair): v = fma(-2, p, B~_j) in FP32 and one compare against a
// per-(row, S tile) threshold tau_i that absorbs every error term; v > tau_i
// proves the FP64 oracle value exceeds T.  The rare remainder gets a per-pair FP64
// certificate: accept (emit), reject, or band (queued for the FP64 refinement
// that reproduces the oracle's summation order).
//
// Warp roles (192 threads, one CTA per SM, persistent over the chunk list):
//   warp 0: TMA producer (one lane), 4-stage ring of {A k-block 16 KB, B k-block 32 KB}
//   warp 1: TMEM allocator + UMMA issuer (one lane), 2 accumulators x 256 columns
//   warps 2-5: epilogue, warp w reads TMEM lanes 32*(w%4) .. +31 (one R row per thread)
#include <cstdio>

#include "tj_emit.cuh"
#include "tj_internal.h"

namespace tj {

namespace {

constexpr int kAccBufs = 2;
constexpr int kEpiWarps = 4;
constexpr int kScreenThreads = (2 + kEpiWarps) * 32;
constexpr unsigned kABytes = kTileR * 128;          // 16 KB
constexpr unsigned kBBytes = kTileS * 128;          // 32 KB
// Stage = one 64-element k-block of A (128 rows) and B (256 rows); with the hi/lo split the
// stage holds both limbs of both operands: [A_hi | A_lo | B_hi | B_lo].
template <int kSplit> struct StageCfg {
    static constexpr unsigned kBytes = (kSplit ? 2u : 1u) * (kABytes + kBBytes);   // 48 or 96 KB
    static constexpr int kStages = kSplit ? 2 : 4;
    static constexpr unsigned kAlo = kABytes;                    // offsets inside a split stage
    static constexpr unsigned kBhi = kSplit ? 2u * kABytes : kABytes;
    static constexpr unsigned kBlo = 2u * kABytes + kBBytes;
};

template <int kStages>
struct ScreenCtl {
    uint64_t full[kStages];
    uint64_t empty[kStages];
    uint64_t acc_full[kAccBufs];
    uint64_t acc_empty[kAccBufs];
    uint64_t drain;
    unsigned tmem_base;
    int abort_flag;
    int acc_ok[2];   // per item parity, like bt: written after the previous item's barrier
    float bt[2][kTileS];
};

template <int kSplit>
constexpr size_t screen_smem() {
    return 1024 + (size_t)StageCfg<kSplit>::kStages * StageCfg<kSplit>::kBytes +
           sizeof(ScreenCtl<StageCfg<kSplit>::kStages>);
}

struct ScreenArgs {
    const uint4* chunks;
    const uint32_t* nchunks;   // device count
    const uint32_t* jlist;
    // R side (rows of tile I)
    const uint32_t* r_row0;
    const uint32_t* r_nvalid;
    const uint32_t* r_perm;
    const double* r_nrm2;
    const float* r_zn;
    const float* r_en;
    const float* r_zl;
    // S side (columns of tile J)
    const uint32_t* s_row0;
    const uint32_t* s_nvalid;
    const uint32_t* s_perm;
    const double* s_nrm2;
    const float* s_nrm2f;
    const float* s_zn;
    const float* s_en;
    const float* s_yn;
    const float* s_zl;
    const float* sJ_maxZl;
    const float* sJ_maxZ;
    const float* sJ_maxE;
    const float* sJ_maxY;
    const float* sJ_maxB;
    const float* sJ_beta;
    int kblocks;
    int kpad;
    unsigned idesc;
    JoinParams jp;
    uint64_t* acc;
    unsigned long long acc_cap;
    uint64_t* band;
    unsigned long long band_cap;
    Counters* ctr;
};

template <int kFmt, int kSplit>   // kFmt: 0 = fp16, 1 = bf16; kSplit: hi/lo operand limbs
__global__ void __launch_bounds__(kScreenThreads, 1)
    screen_tc_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
                     const ScreenArgs a) {
    using Cfg = StageCfg<kSplit>;
    constexpr int kStages = Cfg::kStages;
    constexpr unsigned kStageBytes = Cfg::kBytes;
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    uint8_t* smem = (uint8_t*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    ScreenCtl<kStages>* ctl = (ScreenCtl<kStages>*)(smem + (size_t)kStages * kStageBytes);
    const unsigned warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    unsigned long long* status = &a.ctr->status;

    if (threadIdx.x == 0) {
        for (int s = 0; s < kStages; ++s) {
            mbar_init(&ctl->full[s], 1);
            mbar_init(&ctl->empty[s], 1);
        }
        for (int b = 0; b < kAccBufs; ++b) {
            mbar_init(&ctl->acc_full[b], 1);
            mbar_init(&ctl->acc_empty[b], kEpiWarps);
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
        // ------------------------------------------------------------ TMA producer
        if (lane == 0) {
            unsigned stage = 0, phase = 0;
            bool ok = true;
            for (unsigned c = blockIdx.x; c < nchunks && ok; c += gridDim.x) {
                const uint4 ch = a.chunks[c];
                const int rrow = (int)a.r_row0[ch.x];
                for (unsigned e = ch.y; e < ch.z && ok; ++e) {
                    const int srow = (int)a.s_row0[a.jlist[e]];
                    for (int kb = 0; kb < a.kblocks; ++kb) {
                        if (!mbar_wait(&ctl->empty[stage], phase ^ 1, status)) { ok = false; break; }
                        if (*(volatile int*)&ctl->abort_flag) { ok = false; break; }
                        uint8_t* sa = smem + (size_t)stage * kStageBytes;
                        mbar_arrive_expect_tx(&ctl->full[stage], kStageBytes);
                        tma_load_2d(sa, &tmA, &ctl->full[stage], kb * kBK, rrow);
                        tma_load_2d(sa + Cfg::kBhi, &tmB, &ctl->full[stage], kb * kBK, srow);
                        if (kSplit) {
                            tma_load_2d(sa + Cfg::kAlo, &tmA, &ctl->full[stage], a.kpad + kb * kBK, rrow);
                            tma_load_2d(sa + Cfg::kBlo, &tmB, &ctl->full[stage], a.kpad + kb * kBK, srow);
                        }
                        if (++stage == kStages) { stage = 0; phase ^= 1; }
                    }
                }
            }
            if (!ok) ctl->abort_flag = 1;
            // drain: the last load issued into each stage must have landed before exit
            for (int k = 0; k < kStages; ++k) {
                // stage s was last filled in phase (phase ^ 1) if s >= stage, else in phase `phase`
                const unsigned s = (unsigned)k;
                const unsigned ph = (s < stage) ? phase : (phase ^ 1u);
                mbar_wait(&ctl->full[s], ph, status, 1000000000ull);
            }
        }
    } else if (warp == 1) {
        // ------------------------------------------------------------ UMMA issuer
        if (lane == 0) {
            unsigned stage = 0, phase = 0, acc = 0, acc_phase = 0;
            bool ok = true;
            for (unsigned c = blockIdx.x; c < nchunks && ok; c += gridDim.x) {
                const uint4 ch = a.chunks[c];
                for (unsigned e = ch.y; e < ch.z && ok; ++e) {
                    if (!mbar_wait(&ctl->acc_empty[acc], acc_phase ^ 1, status)) { ok = false; break; }
                    tc_fence_after();
                    const unsigned d_tmem = tmem + acc * kTileS;
                    for (int kb = 0; kb < a.kblocks; ++kb) {
                        if (!mbar_wait(&ctl->full[stage], phase, status)) { ok = false; break; }
                        if (*(volatile int*)&ctl->abort_flag) { ok = false; break; }
                        tc_fence_after();
                        const uint8_t* sa = smem + (size_t)stage * kStageBytes;
#pragma unroll
                        for (int k = 0; k < kBK / 16; ++k) {
                            const uint64_t ad = desc_sw128(sa, k * 32);
                            const uint64_t bd = desc_sw128(sa + Cfg::kBhi, k * 32);
                            umma_f16(d_tmem, ad, bd, a.idesc, (kb | k) != 0 ? 1u : 0u);
                            if (kSplit) {   // z.w ~ hi.hi + hi.lo + lo.hi, one FP32 accumulator
                                umma_f16(d_tmem, ad, desc_sw128(sa + Cfg::kBlo, k * 32), a.idesc, 1u);
                                umma_f16(d_tmem, desc_sw128(sa + Cfg::kAlo, k * 32), bd, a.idesc, 1u);
                            }
                        }
                        umma_commit(&ctl->empty[stage]);
                        if (++stage == kStages) { stage = 0; phase ^= 1; }
                    }
                    if (!ok) break;
                    umma_commit(&ctl->acc_full[acc]);
                    if (++acc == kAccBufs) { acc = 0; acc_phase ^= 1; }
                }
            }
            if (!ok) ctl->abort_flag = 1;
            umma_commit(&ctl->drain);
            mbar_wait(&ctl->drain, 0, status, 1000000000ull);
        }
    } else {
        // ------------------------------------------------------------ epilogue
        const unsigned q = warp & 3;                 // TMEM lane quarter of this warp
        const unsigned et = threadIdx.x - 64;        // 0..127 epilogue thread id
        const unsigned row = q * 32 + lane;          // R row within the tile
        const JoinParams& jp = a.jp;
        WarpAppender app_acc, app_band;
        unsigned acc = 0, acc_phase = 0, par = 0;
        unsigned long long n_screen_acc = 0, n_rare = 0, n_items = 0;
        bool ok = true;
        for (unsigned c = blockIdx.x; c < nchunks && ok; c += gridDim.x) {
            const uint4 ch = a.chunks[c];
            const unsigned I = ch.x;
            const unsigned r0 = a.r_row0[I];
            const bool rvalid = row < a.r_nvalid[I];
            const unsigned rs = r0 + row;
            const double Ai = rvalid ? a.r_nrm2[rs] : 0.0;
            const double Zi = rvalid ? (double)a.r_zn[rs] : 0.0;
            const double Ei = rvalid ? (double)a.r_en[rs] : 0.0;
            const double Zli = rvalid ? (double)a.r_zl[rs] : 0.0;
            for (unsigned e = ch.y; e < ch.z; ++e) {
                const unsigned J = a.jlist[e];
                const unsigned c0 = a.s_row0[J];
                const unsigned nvJ = a.s_nvalid[J];
                ctl->bt[par][et] = et < nvJ ? a.s_nrm2f[c0 + et] : INFINITY;
                ctl->bt[par][et + 128] = et + 128 < nvJ ? a.s_nrm2f[c0 + et + 128] : INFINITY;
                if (et == 0) ctl->acc_ok[par] = mbar_wait(&ctl->acc_full[acc], acc_phase, status) ? 1 : 0;
                asm volatile("bar.sync 1, 128;" ::: "memory");
                if (!ctl->acc_ok[par]) { ok = false; break; }
                tc_fence_after();
                // per-(row, S tile) fast threshold; every error term bounded by tile maxima
                float tau = -INFINITY;
                if (rvalid) {
                    const double WJ = a.sJ_maxZ[J], FJ = a.sJ_maxE[J], YJ = a.sJ_maxY[J];
                    const double BJ = a.sJ_maxB[J], betaJ = a.sJ_beta[J], WlJ = a.sJ_maxZl[J];
                    const double RiJ = jp.gmma * Zi * WJ + jp.cabs + Ei * YJ + Zi * FJ + Zli * WlJ;
                    const double PiJ = Zi * WJ * (1.0 + jp.gmma) + jp.cabs;
                    double t = jp.Tp - Ai + jp.gn * Ai + 0x1p-23 * (BJ + 2.0 * PiJ) + betaJ + 2.0 * RiJ;
                    t = t + fabs(t) * 0x1p-30 + 0x1p-1000;
                    tau = f32_up(t);
                }
                const float* bt = ctl->bt[par];
                const unsigned tbase = tmem + ((q * 32u) << 16) + acc * kTileS;
#pragma unroll 1
                for (int cb = 0; cb < kTileS / 32; ++cb) {
                    uint32_t raw[32];
                    tmem_ld32(tbase + cb * 32, raw);
                    tmem_ld_wait();
                    if (cb == kTileS / 32 - 1) {
                        tc_fence_before();
                        __syncwarp();
                        if (lane == 0) mbar_arrive(&ctl->acc_empty[acc]);
                    }
                    float vmin = INFINITY;
#pragma unroll
                    for (int k = 0; k < 32; ++k)
                        vmin = fminf(vmin, fmaf(-2.f, __uint_as_float(raw[k]), bt[cb * 32 + k]));
                    const bool cand = vmin <= tau;
                    if (!__any_sync(0xffffffffu, cand)) continue;
                    // ---------------- rare path: per-pair FP64 certificate
                    uint32_t amask = 0, bmask = 0;
                    if (cand) {
#pragma unroll
                        for (int k = 0; k < 32; ++k) {
                            const float pk = __uint_as_float(raw[k]);
                            const float v = fmaf(-2.f, pk, bt[cb * 32 + k]);
                            if (v <= tau) {
                                const unsigned col = cb * 32 + k;
                                const unsigned cs = c0 + col;
                                if (jp.self_join && cs <= rs) continue;
                                ++n_rare;
                                const double p = (double)pk;
                                const double Bj = a.s_nrm2[cs];
                                const double Wj = a.s_zn[cs], Fj = a.s_en[cs], Yj = a.s_yn[cs];
                                const double s = Ai + Bj - 2.0 * p;
                                const double R = jp.gmma * Zi * Wj + jp.cabs + Ei * Yj + Zi * Fj +
                                                 Zli * (double)a.s_zl[cs];
                                double m = 2.0 * R + jp.gn * (Ai + Bj) + 0x1p-50 * (Ai + Bj + 2.0 * fabs(p));
                                m = m * (1.0 + 0x1p-40) + 0x1p-1000;
                                if (s + m <= jp.Tm) amask |= 1u << k;
                                else if (!(s - m > jp.Tp)) bmask |= 1u << k;
                            }
                        }
                    }
                    unsigned ta, tb;
                    const unsigned pa = warp_excl_scan(__popc(amask), ta);
                    const unsigned pb = warp_excl_scan(__popc(bmask), tb);
                    if (ta) {
                        const unsigned long long base = app_acc.reserve(ta, &a.ctr->acc_reserved, a.acc, a.acc_cap);
                        unsigned long long pos = base + pa;
                        uint32_t mk = amask;
                        while (mk) {
                            const int k = __ffs(mk) - 1;
                            mk &= mk - 1;
                            const unsigned cs = c0 + cb * 32 + k;
                            if (pos < a.acc_cap) a.acc[pos] = pair_key(jp, a.r_perm[rs], a.s_perm[cs]);
                            ++pos;
                        }
                        n_screen_acc += __popc(amask);
                    }
                    if (tb) {
                        const unsigned long long base =
                            app_band.reserve(tb, &a.ctr->band_reserved, a.band, a.band_cap);
                        unsigned long long pos = base + pb;
                        uint32_t mk = bmask;
                        while (mk) {
                            const int k = __ffs(mk) - 1;
                            mk &= mk - 1;
                            const unsigned cs = c0 + cb * 32 + k;
                            if (pos < a.band_cap) a.band[pos] = pair_key(jp, a.r_perm[rs], a.s_perm[cs]);
                            ++pos;
                        }
                    }
                }
                ++n_items;
                par ^= 1;
                if (++acc == kAccBufs) { acc = 0; acc_phase ^= 1; }
            }
        }
        if (!ok) ctl->abort_flag = 1;
        app_acc.pad(a.acc, a.acc_cap);
        app_band.pad(a.band, a.band_cap);
        // warp totals
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            n_screen_acc += __shfl_xor_sync(0xffffffffu, n_screen_acc, o);
            n_rare += __shfl_xor_sync(0xffffffffu, n_rare, o);
        }
        if (lane == 0) {
            if (app_acc.valid) atomicAdd(&a.ctr->acc_valid, app_acc.valid);
            if (app_band.valid) atomicAdd(&a.ctr->band_valid, app_band.valid);
            if (n_screen_acc) atomicAdd(&a.ctr->screen_accept, n_screen_acc);
            if (n_rare) atomicAdd(&a.ctr->rare_checks, n_rare);
            if (q == 0 && n_items) atomicAdd(&a.ctr->items, n_items);
        }
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (warp == 1) tmem_dealloc(tmem, 512);
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
void make_tmap_2d(CUtensorMap* m, const void* base, long long rows, long long cols, int esize, int box_rows,
                  CUtensorMapDataType dt) {
    const cuuint64_t dims[2] = {(cuuint64_t)cols, (cuuint64_t)rows};
    const cuuint64_t strides[1] = {(cuuint64_t)cols * esize};
    const cuuint32_t box[2] = {(cuuint32_t)(128 / esize), (cuuint32_t)box_rows};
    const cuuint32_t estr[2] = {1, 1};
    const CUresult r = encode_fn()(m, dt, 2, const_cast<void*>(base), dims, strides, box, estr,
                                   CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                                   CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) fail(-2, "cuTensorMapEncodeTiled failed (" + std::to_string((int)r) + ")");
}

void screen_tc(const JoinGeometry& g, const EmitBuffers& eb, cudaStream_t st) {
    const Side& R = *g.R;
    const Side& S = *g.S;
    const bool bf = R.screen == kScreenBF16 || R.screen == kScreenBF16X3;
    const bool ok = R.screen == S.screen && (bf || R.screen == kScreenFP16 || R.screen == kScreenFP16X3);
    if (!ok) fail(-1, "screen_tc needs matching bf16 / fp16 operands on both sides");
    if (R.kpad != S.kpad || R.split != S.split) fail(-1, "operand layouts differ");
    CUtensorMap tmA, tmB;
    const CUtensorMapDataType dt = bf ? CU_TENSOR_MAP_DATA_TYPE_BFLOAT16 : CU_TENSOR_MAP_DATA_TYPE_FLOAT16;
    const long long w = (long long)R.kpad * (R.split ? 2 : 1);
    make_tmap_2d(&tmA, R.op.p, R.rows_pad, w, 2, kTileR, dt);
    make_tmap_2d(&tmB, S.op.p, S.rows_pad, w, 2, kTileS, dt);
    ScreenArgs a;
    a.chunks = g.cand->chunks.p;
    a.nchunks = g.cand->dev_counts.p + 1;
    a.jlist = g.cand->jlist.p;
    a.r_row0 = g.tR->row0.p;
    a.r_nvalid = g.tR->nvalid.p;
    a.r_perm = R.perm.p;
    a.r_nrm2 = R.nrm2.p;
    a.r_zn = R.zn.p;
    a.r_en = R.en.p;
    a.r_zl = R.zl.p;
    a.s_row0 = g.tS->row0.p;
    a.s_nvalid = g.tS->nvalid.p;
    a.s_perm = S.perm.p;
    a.s_nrm2 = S.nrm2.p;
    a.s_nrm2f = S.nrm2f.p;
    a.s_zn = S.zn.p;
    a.s_en = S.en.p;
    a.s_yn = S.yn.p;
    a.s_zl = S.zl.p;
    a.sJ_maxZl = g.tS->maxZl.p;
    a.sJ_maxZ = g.tS->maxZ.p;
    a.sJ_maxE = g.tS->maxE.p;
    a.sJ_maxY = g.tS->maxY.p;
    a.sJ_maxB = g.tS->maxB.p;
    a.sJ_beta = g.tS->beta.p;
    a.kblocks = R.kpad / kBK;
    a.kpad = R.kpad;
    a.idesc = make_idesc(1u, bf ? 1u : 0u, kTileR, kTileS);
    a.jp = g.jp;
    a.acc = eb.acc;
    a.acc_cap = eb.acc_cap;
    a.band = eb.band;
    a.band_cap = eb.band_cap;
    a.ctr = eb.ctr;
    const int grid = num_sms();
#define TJ_SCREEN(F, SP)                                                                                    \
    do {                                                                                                    \
        TJ_CUDA(cudaFuncSetAttribute(screen_tc_kernel<F, SP>, cudaFuncAttributeMaxDynamicSharedMemorySize, \
                                     (int)screen_smem<SP>()));                                              \
        launch(screen_tc_kernel<F, SP>, grid, kScreenThreads, screen_smem<SP>(), st, tmA, tmB, a);          \
    } while (0)
    if (bf && R.split) TJ_SCREEN(1, 1);
    else if (bf) TJ_SCREEN(1, 0);
    else if (R.split) TJ_SCREEN(0, 1);
    else TJ_SCREEN(0, 0);
#undef TJ_SCREEN
}

}  // namespace tj
