// FP64 band refinement, the plain FP32 direct-difference join, and the
// canonical-output helpers (directed expansion, pair decoding).
//
// Refinement reproduces the oracle's predicate exactly: for every band pair,
//   acc = 0; for k = 0..d-1: t = dbl(x_k) - dbl(y_k); acc = acc + t*t   (one rounding each, no FMA)
//   accept iff acc <= T
// which is the reference's FP64 terminal (src/run_g2a_tensorjoin.py:194-232,
// src/run_d1_triton.py:206-248) with its summation order fixed to sequential k
// (the reference summed 256-wide blocks in tree order), so the emitted pair set is
// bit-identical to the CPU oracle.
//
// The plain join is the "plain GPU method" baseline: FP32 direct difference over
// the same candidate tile pairs (no tensor cores), a rigorous FP32 error band, and
// the same FP64 refinement of band pairs.  It plays the role of the reference's
// GDS-Join FP64 grid join / FP32-first control (adapters/gds_g2a/kernel.cu:314-386,
// g15_strong_control_20260905/src/fp32_first.py:104-157).
#include <cstring>
#include <vector>

#include "tj_emit.cuh"
#include "tj_internal.h"

namespace tj {

namespace {

// ------------------------------------------------------------------ plain FP32 join
constexpr int kPT = 256;                // threads: 16 x 16
constexpr int kPR = 8, kPC = 16;        // micro-tile: 8 rows x 16 cols per thread
constexpr int kPK = 16;                 // k chunk

struct PlainClass {
    const float* rx;     // [rows_pad, d] sorted FP32 rows (R side of the class)
    const float* sx;     // [rows_pad, d] sorted FP32 rows (S side)
    const uint32_t* r_emit;
    const uint32_t* s_emit;
    int d;
};

struct PlainArgs {
    const uint4* chunks;
    const uint32_t* nchunks;
    const uint32_t* jlist;
    const uint4* rtiles;        // (row0, nvalid, join, class) per global R tile
    const uint4* stiles;
    const JoinParams* jps;
    const float2* thr;          // per join: certified-in / certified-out thresholds on the FP32 sum
    PlainClass cls[kMaxClass];
    uint64_t* acc;
    unsigned long long acc_cap;
    uint64_t* band;
    unsigned long long band_cap;
    Counters* ctr;
};

// a0 += (r - s0)^2, a1 += (r - s1)^2 as one packed FP32x2 subtract and one packed FP32x2 FMA (sm_100);
// each lane is rounded exactly as the scalar subtract and fmaf
TJ_DEV void sqdiff_acc_x2(float r, float s0, float s1, float& a0, float& a1) {
    asm("{\n\t.reg .b64 x, y, t, c;\n\t"
        "mov.b64 x, {%2, %2};\n\t"
        "mov.b64 y, {%3, %4};\n\t"
        "mov.b64 c, {%0, %1};\n\t"
        "sub.rn.f32x2 t, x, y;\n\t"
        "fma.rn.f32x2 c, t, t, c;\n\t"
        "mov.b64 {%0, %1}, c;\n\t}"
        : "+f"(a0), "+f"(a1) : "f"(r), "f"(s0), "f"(s1));
}

__global__ void __launch_bounds__(kPT, 1) plain_kernel(const PlainArgs a) {
    __shared__ float sR[kPK][kTileR + 1];   // +1: conflict-free transposed stores
    __shared__ float sS[kPK][kTileS + 1];
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
    const unsigned nchunks = *a.nchunks;
    WarpAppender app_acc, app_band;
    unsigned long long n_items = 0, n_screen_acc = 0;
    for (unsigned c = blockIdx.x; c < nchunks; c += gridDim.x) {
        const uint4 ch = a.chunks[c];
        const uint4 rt = a.rtiles[ch.x];
        const PlainClass& pc = a.cls[rt.w];
        const JoinParams jp = a.jps[rt.z];
        const float2 th = a.thr[rt.z];
        const int d = pc.d;
        const unsigned r0 = rt.x, nvI = rt.y;
        for (unsigned e = ch.y; e < ch.z; ++e) {
            const unsigned J = a.jlist[e];
            const uint4 stt = a.stiles[J];
            const unsigned c0 = stt.x, nvJ = stt.y;
            float acc[kPR][kPC];
#pragma unroll
            for (int i = 0; i < kPR; ++i)
#pragma unroll
                for (int j = 0; j < kPC; ++j) acc[i][j] = 0.f;
            for (int k0 = 0; k0 < d; k0 += kPK) {
                __syncthreads();
                for (int idx = threadIdx.x; idx < kPK * kTileR; idx += kPT) {
                    const int r = idx / kPK, k = idx % kPK;
                    sR[k][r] = (k0 + k < d) ? pc.rx[(size_t)(r0 + r) * d + k0 + k] : 0.f;
                }
                for (int idx = threadIdx.x; idx < kPK * kTileS; idx += kPT) {
                    const int r = idx / kPK, k = idx % kPK;
                    sS[k][r] = (k0 + k < d) ? pc.sx[(size_t)(c0 + r) * d + k0 + k] : 0.f;
                }
                __syncthreads();
                const int kmax = min(kPK, d - k0);
                for (int k = 0; k < kmax; ++k) {
                    float rv[kPR], sv[kPC];
#pragma unroll
                    for (int i = 0; i < kPR; ++i) rv[i] = sR[k][i * 16 + ty];   // rows i*16+ty, cols j*16+tx
#pragma unroll
                    for (int j = 0; j < kPC; ++j) sv[j] = sS[k][j * 16 + tx];
#pragma unroll
                    for (int i = 0; i < kPR; ++i)
#pragma unroll
                        for (int j = 0; j < kPC; j += 2)
                            sqdiff_acc_x2(rv[i], sv[j], sv[j + 1], acc[i][j], acc[i][j + 1]);
                }
            }
            // classify: groups of 32 pairs (2 rows x 16 cols) so that emission stays warp-uniform
#pragma unroll
            for (int g = 0; g < kPR / 2; ++g) {
                uint32_t amask = 0, bmask = 0;
#pragma unroll
                for (int h = 0; h < 2; ++h)
#pragma unroll
                    for (int j = 0; j < kPC; ++j) {
                        const int i = g * 2 + h;
                        const unsigned row = i * 16 + ty, col = j * 16 + tx;
                        const float s = acc[i][j];
                        if (s > th.y || row >= nvI || col >= nvJ) continue;
                        if (jp.self_join && c0 + col <= r0 + row) continue;
                        if (s <= th.x) amask |= 1u << (h * 16 + j);
                        else bmask |= 1u << (h * 16 + j);
                    }
                unsigned ta, tb;
                const unsigned pa = warp_excl_scan(__popc(amask), ta);
                const unsigned pb = warp_excl_scan(__popc(bmask), tb);
                if (ta) {
                    unsigned long long pos = app_acc.reserve(ta, &a.ctr->acc_reserved, a.acc, a.acc_cap) + pa;
                    uint32_t mk = amask;
                    while (mk) {
                        const int b = __ffs(mk) - 1;
                        mk &= mk - 1;
                        const unsigned row = (g * 2 + (b >> 4)) * 16 + ty, col = (b & 15) * 16 + tx;
                        if (pos < a.acc_cap) a.acc[pos] = pair_key(jp, pc.r_emit[r0 + row], pc.s_emit[c0 + col]);
                        ++pos;
                    }
                    n_screen_acc += __popc(amask);
                }
                if (tb) {
                    unsigned long long pos = app_band.reserve(tb, &a.ctr->band_reserved, a.band, a.band_cap) + pb;
                    uint32_t mk = bmask;
                    while (mk) {
                        const int b = __ffs(mk) - 1;
                        mk &= mk - 1;
                        const unsigned row = (g * 2 + (b >> 4)) * 16 + ty, col = (b & 15) * 16 + tx;
                        if (pos < a.band_cap) a.band[pos] = pair_key(jp, pc.r_emit[r0 + row], pc.s_emit[c0 + col]);
                        ++pos;
                    }
                }
            }
            ++n_items;
        }
    }
    app_acc.pad(a.acc, a.acc_cap);
    app_band.pad(a.band, a.band_cap);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) n_screen_acc += __shfl_xor_sync(0xffffffffu, n_screen_acc, o);
    if (lane_id() == 0) {
        if (app_acc.valid) atomicAdd(&a.ctr->acc_valid, app_acc.valid);
        if (app_band.valid) atomicAdd(&a.ctr->band_valid, app_band.valid);
        if (n_screen_acc) atomicAdd(&a.ctr->screen_accept, n_screen_acc);
        if (threadIdx.x == 0 && n_items) atomicAdd(&a.ctr->items, n_items);
    }
}

// ------------------------------------------------------------------ FP64 refinement
struct RefineArgs {
    const uint64_t* band;
    unsigned long long band_cap;
    const JoinParams* jps;              // per join
    const unsigned long long* key_off;  // ascending key offset of each join
    int njoins;
    const void* const* rsrc;            // caller's rows of each join, original order
    const void* const* ssrc;
    uint64_t* acc;
    unsigned long long acc_cap;
    Counters* ctr;
    const float2* thr;                  // per join FP32-sum thresholds (the FP32 band stage)
    int is_int;                         // int16 (int14) rows: exact integer distances against T_int
    long long T_int;
};

// FP32 sum of squared FP32 differences in four FMA chains (tree depth <= d / 4 + 2), the FP32
// band stage's value; certified against the FP64 oracle by fp32_sum_thresholds.
TJ_DEV float fp32_d2(const float* x, const float* y, int d) {
    float a0 = 0.f, a1 = 0.f, a2 = 0.f, a3 = 0.f;
    if ((d & 3) == 0 && ((((uintptr_t)x) | ((uintptr_t)y)) & 15) == 0) {
        const float4* x4 = (const float4*)x;
        const float4* y4 = (const float4*)y;
        for (int k = 0; k < d / 4; ++k) {
            const float4 a = __ldg(x4 + k), b = __ldg(y4 + k);
            float t;
            t = a.x - b.x; a0 = fmaf(t, t, a0);
            t = a.y - b.y; a1 = fmaf(t, t, a1);
            t = a.z - b.z; a2 = fmaf(t, t, a2);
            t = a.w - b.w; a3 = fmaf(t, t, a3);
        }
    } else {
        for (int k = 0; k < d; ++k) {
            const float t = __ldg(x + k) - __ldg(y + k);
            a0 = fmaf(t, t, a0);
        }
    }
    return (a0 + a1) + (a2 + a3);
}

TJ_DEV double seq_d2(const float* x, const float* y, int d) {
    double acc = 0.0;
    if ((d & 3) == 0 && ((((uintptr_t)x) | ((uintptr_t)y)) & 15) == 0) {
        const float4* x4 = (const float4*)x;
        const float4* y4 = (const float4*)y;
        for (int k = 0; k < d / 4; ++k) {
            const float4 a = __ldg(x4 + k), b = __ldg(y4 + k);
            double t;
            t = __dsub_rn((double)a.x, (double)b.x); acc = __dadd_rn(acc, __dmul_rn(t, t));
            t = __dsub_rn((double)a.y, (double)b.y); acc = __dadd_rn(acc, __dmul_rn(t, t));
            t = __dsub_rn((double)a.z, (double)b.z); acc = __dadd_rn(acc, __dmul_rn(t, t));
            t = __dsub_rn((double)a.w, (double)b.w); acc = __dadd_rn(acc, __dmul_rn(t, t));
        }
    } else {
        for (int k = 0; k < d; ++k) {
            const double t = __dsub_rn((double)__ldg(x + k), (double)__ldg(y + k));
            acc = __dadd_rn(acc, __dmul_rn(t, t));
        }
    }
    return acc;
}

// Exact squared distance of two int16 rows in int64: each difference fits int32 and its square
// int64, so no order of the sum can round (the oracle's exact integer predicate).
TJ_DEV long long exact_d2_i16(const int16_t* x, const int16_t* y, int d) {
    long long acc = 0;
    if ((d & 7) == 0 && ((((uintptr_t)x) | ((uintptr_t)y)) & 15) == 0) {
        const int4* x4 = (const int4*)x;
        const int4* y4 = (const int4*)y;
        for (int k = 0; k < d / 8; ++k) {
            const int4 a = __ldg(x4 + k), b = __ldg(y4 + k);
            const int av[4] = {a.x, a.y, a.z, a.w}, bv[4] = {b.x, b.y, b.z, b.w};
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const int t0 = (int)(short)(av[u] & 0xffff) - (int)(short)(bv[u] & 0xffff);
                const int t1 = (av[u] >> 16) - (bv[u] >> 16);
                acc += (long long)t0 * t0 + (long long)t1 * t1;
            }
        }
    } else {
        for (int k = 0; k < d; ++k) {
            const int t = (int)__ldg(x + k) - (int)__ldg(y + k);
            acc += (long long)t * t;
        }
    }
    return acc;
}

// Band pairs -> accept buffer.  kFp32: each pair is first decided, where it can be, by the
// certified FP32 sum (the FP32 band stage); only the rest pay the sequential FP64 terminal.
template <bool kFp32>
__global__ void refine_kernel(const RefineArgs a) {
    const unsigned long long n = min(a.ctr->band_reserved, a.band_cap);
    const unsigned long long stride = (unsigned long long)gridDim.x * blockDim.x;
    const unsigned long long start = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x;
    unsigned long long n_acc = 0, n_fp64 = 0;
    // loop count is warp-uniform so the ballot below is well formed
    const unsigned long long warp_start = start & ~31ull;
    for (unsigned long long w = warp_start; w < n; w += stride) {
        const unsigned long long idx = w + lane_id();
        bool ok = false;
        uint64_t key = kSentinel;
        if (idx < n) {
            key = a.band[idx];
            if (key != kSentinel) {
                int lo = 0, hi = a.njoins - 1;   // join owning the key: last offset <= key
                while (lo < hi) {
                    const int mid = (lo + hi + 1) >> 1;
                    if (a.key_off[mid] <= key) lo = mid; else hi = mid - 1;
                }
                const JoinParams& jp = a.jps[lo];
                const uint64_t local = key - jp.key_off;
                const uint64_t i = local / (uint64_t)jp.n_cols, j = local - i * (uint64_t)jp.n_cols;
                if (i >= (uint64_t)jp.n_rows) {   // not a key the screen wrote: flagged, no row is read
                    atomicOr(&a.ctr->status, (unsigned long long)kStatusGuard);
                } else if (a.is_int) {   // int14 rows: the exact integer predicate decides every pair
                    const int16_t* xi = (const int16_t*)a.rsrc[lo] + (size_t)i * jp.d;
                    const int16_t* yi = (const int16_t*)a.ssrc[lo] + (size_t)j * jp.d;
                    ok = exact_d2_i16(xi, yi, jp.d) <= a.T_int;
                } else {
                const float* x = (const float*)a.rsrc[lo] + (size_t)i * jp.d;
                const float* y = (const float*)a.ssrc[lo] + (size_t)j * jp.d;
                bool decided = false;
                if (kFp32) {
                    const float s = fp32_d2(x, y, jp.d);
                    const float2 th = a.thr[lo];
                    if (s <= th.x) { ok = true; decided = true; }
                    else if (s > th.y) { decided = true; }
                }
                if (!decided) {
                    ok = seq_d2(x, y, jp.d) <= jp.T;
                    ++n_fp64;
                }
                }
            }
        }
        const unsigned m = __ballot_sync(0xffffffffu, ok);
        if (m) {
            unsigned long long base = 0;
            if (lane_id() == 0) base = atomicAdd(&a.ctr->acc_reserved, (unsigned long long)__popc(m));
            base = __shfl_sync(0xffffffffu, base, 0);
            if (ok) {
                const unsigned long long pos = base + __popc(m & ((1u << lane_id()) - 1u));
                if (pos < a.acc_cap) a.acc[pos] = key;
            }
            n_acc += (lane_id() == 0) ? __popc(m) : 0;
        }
    }
    if (lane_id() == 0 && n_acc) {
        atomicAdd(&a.ctr->acc_valid, n_acc);
        atomicAdd(&a.ctr->refine_accept, n_acc);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) n_fp64 += __shfl_xor_sync(0xffffffffu, n_fp64, o);
    if (lane_id() == 0 && n_fp64) atomicAdd(&a.ctr->band_fp64, n_fp64);
}

// ------------------------------------------------------------------ canonical output helpers
__global__ void expand_directed_kernel(const uint64_t* upper, unsigned long long slots, uint64_t* out, long long N) {
    const unsigned long long i = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < slots) {
        const uint64_t k = upper[i];
        out[2 * i] = k;
        if (k == kSentinel) {
            out[2 * i + 1] = kSentinel;
        } else {
            const uint64_t lo = k / (uint64_t)N, hi = k - lo * (uint64_t)N;
            out[2 * i + 1] = hi * (uint64_t)N + lo;
        }
    }
    if (i < (unsigned long long)N) out[2 * slots + i] = i * (uint64_t)N + i;
}

__global__ void decode_kernel(const uint64_t* keys, long long n, long long n_cols, int64_t* io, int64_t* jo) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const uint64_t k = keys[t];
    const uint64_t i = k / (uint64_t)n_cols;
    io[t] = (int64_t)i;
    jo[t] = (int64_t)(k - i * (uint64_t)n_cols);
}

__global__ void decode_batched_kernel(const uint64_t* keys, long long n, const unsigned long long* key_off,
                                     const long long* n_cols, int njoins, int64_t* io, int64_t* jo) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const uint64_t k = keys[t];
    int lo = 0, hi = njoins - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (key_off[mid] <= k) lo = mid; else hi = mid - 1;
    }
    const uint64_t local = k - key_off[lo];
    const uint64_t i = local / (uint64_t)n_cols[lo];
    io[t] = (int64_t)i;
    jo[t] = (int64_t)(local - i * (uint64_t)n_cols[lo]);
}

// offsets[k] = first position of a key >= key_off[k] in the sorted keys; offsets[njoins] = n.
__global__ void batch_offsets_kernel(const uint64_t* keys, long long n, const unsigned long long* key_off,
                                     int njoins, long long* offsets) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k > njoins) return;
    if (k == njoins) { offsets[k] = n; return; }
    long long lo = 0, hi = n;
    const uint64_t v = key_off[k];
    while (lo < hi) {
        const long long mid = (lo + hi) >> 1;
        if (keys[mid] < v) lo = mid + 1; else hi = mid;
    }
    offsets[k] = lo;
}

}  // namespace

// Per join, thresholds on an FP32 sum s of the d squared FP32 differences (FMA accumulation, any
// summation tree of depth <= d + 2): s <= x certifies the FP64 oracle value <= T, s > y certifies
// it > T.  |s - D| <= gamma_{d+4} D + (d + 4) 2^-147 with u = 2^-24 (one rounding in each
// difference, one in each FMA or add along the tree, subnormal products absolutely).
static void fp32_sum_thresholds(const ScreenInput& g, float2* dst, cudaStream_t st) {
    const JoinParams* hj = g.h_jps;
    if (!hj) fail(-1, "the FP32 thresholds need the host join parameters");
    std::vector<float2> th((size_t)g.njoins);
    for (int k = 0; k < g.njoins; ++k) {
        const double u = 0x1p-24, nu = (double)(hj[k].d + 4) * u;
        const double gam = nu / (1.0 - nu);
        const double tiny = (double)(hj[k].d + 4) * 0x1p-147;
        const double tin = (hj[k].Tm - tiny) * (1.0 - gam) * (1.0 - 0x1p-30);
        const double tout = (hj[k].Tp + tiny) * (1.0 + gam) * (1.0 + 0x1p-30) + tiny;
        float fin = tin > 0 ? (float)tin : -1.f;   // nearest, then nudged to stay a lower bound
        if (fin > 0 && (double)fin > tin) fin = nextafterf(fin, 0.f);
        float fout = (float)tout;
        if ((double)fout < tout) fout = nextafterf(fout, INFINITY);
        th[k] = make_float2(fin, fout);
    }
    upload(dst, th.data(), g.njoins * sizeof(float2), st);
}

void screen_plain(const ScreenInput& g, const EmitBuffers& eb, cudaStream_t st) {
    PlainArgs a;
    memset(&a, 0, sizeof(a));
    for (int c = 0; c < g.ncls; ++c) {
        const Side& R = *g.R[c];
        const Side& S = *g.S[c];
        if (R.screen != kScreenPlain || S.screen != kScreenPlain) fail(-1, "screen_plain needs FP32 sides");
        a.cls[c].rx = R.xs.p;
        a.cls[c].sx = S.xs.p;
        a.cls[c].r_emit = R.emit;
        a.cls[c].s_emit = S.emit;
        a.cls[c].d = R.d;
    }
    DBuf<float2> dth((size_t)g.njoins, st);
    fp32_sum_thresholds(g, dth.p, st);
    a.chunks = g.cand->chunks.p;
    a.nchunks = g.cand->dev_counts.p + 1;
    a.jlist = g.cand->jlist.p;
    a.rtiles = g.rtiles;
    a.stiles = g.stiles;
    a.jps = g.jps;
    a.thr = dth.p;
    a.acc = eb.acc;
    a.acc_cap = eb.acc_cap;
    a.band = eb.band;
    a.band_cap = eb.band_cap;
    a.ctr = eb.ctr;
    launch(plain_kernel, num_sms() * 2, kPT, 0, st, a);
}

void refine_band(const ScreenInput& g, const EmitBuffers& eb, bool fp32_stage, cudaStream_t st) {
    RefineArgs a;
    a.band = eb.band;
    a.band_cap = eb.band_cap;
    a.jps = g.jps;
    a.key_off = g.key_off;
    a.njoins = g.njoins;
    a.rsrc = g.rsrc;
    a.ssrc = g.ssrc;
    a.acc = eb.acc;
    a.acc_cap = eb.acc_cap;
    a.ctr = eb.ctr;
    a.thr = nullptr;
    a.is_int = g.R[0]->dtype == kI16 ? 1 : 0;
    a.T_int = g.T_int;
    if (a.is_int && g.njoins != 1) fail(-7, "int16 band refinement runs one join at a time");
    if (fp32_stage && !a.is_int) {
        DBuf<float2> dth((size_t)g.njoins, st);
        fp32_sum_thresholds(g, dth.p, st);
        a.thr = dth.p;
        launch(refine_kernel<true>, num_sms() * 8, 256, 0, st, a);
    } else {
        launch(refine_kernel<false>, num_sms() * 8, 256, 0, st, a);
    }
}

void expand_directed(const uint64_t* upper, unsigned long long slots, uint64_t* out, long long N, cudaStream_t st) {
    const unsigned long long n = slots > (unsigned long long)N ? slots : (unsigned long long)N;
    if (n == 0) return;
    launch(expand_directed_kernel, (unsigned)((n + 255) / 256), 256, 0, st, upper, slots, out, N);
    TJ_CUDA(cudaGetLastError());
}

void decode_pairs_batched(const uint64_t* keys, long long n, const unsigned long long* key_off,
                          const long long* n_cols, int njoins, int64_t* i_out, int64_t* j_out, cudaStream_t st) {
    if (n <= 0) return;
    launch(decode_batched_kernel, (unsigned)((n + 255) / 256), 256, 0, st, keys, n, key_off, n_cols, njoins, i_out,
           j_out);
}

void batch_offsets(const uint64_t* keys, long long n, const unsigned long long* key_off, int njoins,
                   long long* offsets, cudaStream_t st) {
    launch(batch_offsets_kernel, (unsigned)((njoins + 1 + 255) / 256), 256, 0, st, keys, n, key_off, njoins, offsets);
}

void decode_pairs(const uint64_t* keys, long long n, long long n_cols, int64_t* i_out, int64_t* j_out,
                  cudaStream_t st) {
    if (n <= 0) return;
    launch(decode_kernel, (unsigned)((n + 255) / 256), 256, 0, st, keys, n, n_cols, i_out, j_out);
    TJ_CUDA(cudaGetLastError());
}

}  // namespace tj
