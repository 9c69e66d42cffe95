// C ABI of libtensorjoin: orchestration of index -> candidates -> screen -> refine -> sort.
//
// One host synchronisation per join: after the screen and the refinement the
// counters are read back once to size the output (and to detect a capacity
// overflow, in which case both stages run again with larger buffers -- the
// overflow-and-retry pass of the reference, src/run_g2a_tensorjoin.py:329-378).
// Everything else stays on the device in stream order; memory comes from a
// private stream-ordered pool so repeated joins do not hit cudaMalloc.
#include <algorithm>
#include <chrono>
#include <atomic>
#include <cmath>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>

#include "../../include/tensorjoin.h"
#include "tj_internal.h"

namespace tj {

// ------------------------------------------------------------------ errors
namespace {
thread_local std::string g_last_error;
}

void fail(int code, const std::string& msg) { throw Error{code, msg}; }
void set_last_error(const std::string& msg) { g_last_error = msg; }

void check_cuda(cudaError_t e, const char* what) {
    if (e == cudaSuccess) return;
    const int code = (e == cudaErrorMemoryAllocation) ? TJ_ERR_NOMEM : TJ_ERR_CUDA;
    fail(code, std::string(what) + ": " + cudaGetErrorString(e));
}

namespace {
int g_sms[64] = {};
}  // namespace

namespace {
std::atomic<long long> g_launches{0};
thread_local unsigned long long g_wait_ns = kWaitLimitNs;   // pipeline wait limit of this thread's joins
}
void count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }
unsigned long long pipeline_wait_ns() { return g_wait_ns; }

namespace {
struct StageChunk {
    uint8_t* p = nullptr;
    size_t cap = 0, used = 0;
};
thread_local std::vector<StageChunk> g_stage;
thread_local cudaEvent_t g_stage_done = nullptr;   // recorded after the latest staged copy
thread_local bool g_stage_pending = false;
}  // namespace

// Makes every staging region reusable.  Waits for the last staged copy first (a call that failed
// part-way may have left one in flight); on the normal path the join already synchronised, so the
// wait returns at once.
void stage_reset() {
    if (g_stage_pending) {
        TJ_CUDA(cudaEventSynchronize(g_stage_done));
        g_stage_pending = false;
    }
    for (auto& c : g_stage) c.used = 0;
}

void upload(void* dev_dst, const void* host_src, size_t bytes, cudaStream_t st) {
    if (bytes == 0) return;
    const size_t need = (bytes + 255) & ~(size_t)255;
    StageChunk* ch = nullptr;
    for (auto& c : g_stage)
        if (c.cap - c.used >= need) { ch = &c; break; }
    if (!ch) {
        StageChunk c;
        c.cap = std::max<size_t>(need, (size_t)4 << 20);
        TJ_CUDA(cudaMallocHost((void**)&c.p, c.cap));
        g_stage.push_back(c);
        ch = &g_stage.back();
    }
    uint8_t* src = ch->p + ch->used;
    ch->used += need;
    memcpy(src, host_src, bytes);
    TJ_CUDA(cudaMemcpyAsync(dev_dst, src, bytes, cudaMemcpyHostToDevice, st));
    if (!g_stage_done) TJ_CUDA(cudaEventCreateWithFlags(&g_stage_done, cudaEventDisableTiming));
    TJ_CUDA(cudaEventRecord(g_stage_done, st));
    g_stage_pending = true;
}

int num_sms() {
    int dev = 0;
    TJ_CUDA(cudaGetDevice(&dev));
    if (!g_sms[dev]) TJ_CUDA(cudaDeviceGetAttribute(&g_sms[dev], cudaDevAttrMultiProcessorCount, dev));
    return g_sms[dev];
}

// ------------------------------------------------------------------ helpers
namespace {

struct ScreenOps {
    unsigned long long per_pair[kMaxClass];   // algorithmic operations per screened pair
    double per_item[kMaxClass];               // tensor-core operations issued per tile pair
};

__global__ void zero_counters(Counters* c, int emit_only) {
    unsigned long long* w = (unsigned long long*)c;
    const int n = emit_only ? kCountersPerAttempt : (int)(sizeof(Counters) / 8);
    for (int i = threadIdx.x; i < n; i += blockDim.x) w[i] = 0;
}

// Guard regions (TJ_FLAG_GUARDS): kGuardSlots words of a fixed pattern written right after the
// part of an output buffer a stage may write, and checked after the stage.  The pattern is -17 in
// every byte, the reference's fill for its retained buffers.
constexpr unsigned long long kGuardSlots = 512;
constexpr uint64_t kGuardWord = 0xEFEFEFEFEFEFEFEFull;
__global__ void guard_fill(uint64_t* p) {
    for (unsigned i = threadIdx.x; i < kGuardSlots; i += blockDim.x) p[i] = kGuardWord;
}
__global__ void guard_check(const uint64_t* p, Counters* c) {
    bool bad = false;
    for (unsigned i = threadIdx.x; i < kGuardSlots; i += blockDim.x) bad |= p[i] != kGuardWord;
    if (__syncthreads_or(bad) && threadIdx.x == 0) atomicOr(&c->status, (unsigned long long)kStatusGuard);
}
__global__ void snapshot_reserved(Counters* c) { c->screen_reserved = c->acc_reserved; }

__global__ void cell_flags(const uint64_t* keys, long long n, uint32_t* flag) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) flag[i] = (i == 0 || keys[i] != keys[i - 1]) ? 1u : 0u;
}
__global__ void cell_starts(const uint32_t* flag, const uint32_t* pos, long long n, uint32_t* start,
                            const uint32_t* ncells) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n && flag[i]) start[pos[i]] = (uint32_t)i;
    if (i == 0) start[*ncells] = (uint32_t)n;
}
// Distance evaluations of the candidate list (out[0] = pairs_screened), algorithmic screen operations
// (out[1], ops_per_pair[c] = 2 d (16-bit), 6 d (hi/lo split) or 8 d (int8 limbs) for class c) and tile
// pairs per class (out[2 + c] = class_items[c], for the issued-operation count).
__global__ void pairs_screened_kernel(const uint4* chunks, const uint32_t* nchunks, const uint32_t* jlist,
                                      const uint4* rtiles, const uint4* stiles, const ScreenOps ops, int half,
                                      unsigned long long* out) {
    unsigned long long acc = 0, aops = 0, items[kMaxClass] = {0, 0, 0, 0};
    const unsigned n = *nchunks;
    for (unsigned c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x) {
        const uint4 ch = chunks[c];
        const uint4 rt = rtiles[ch.x];
        const unsigned long long rv = rt.y;
        unsigned long long p = 0, hi = 0;   // hi: 128-column half-items issued
        for (unsigned e = ch.y; e < ch.z; ++e) {
            const uint32_t je = jlist[e];
            const unsigned nv = stiles[je & kJMask].y;
            if (!half) {
                p += rv * nv;
                hi += 2;
                continue;
            }
            const unsigned m = je >> 30;
            if (m & 1u) { p += rv * min(nv, 128u); ++hi; }
            if (m & 2u) { p += rv * (nv > 128u ? nv - 128u : 0u); ++hi; }
        }
        acc += p;
        aops += p * ops.per_pair[rt.w];
#pragma unroll
        for (int q = 0; q < kMaxClass; ++q) items[q] += rt.w == (unsigned)q ? hi : 0u;
    }
    for (int o = 16; o > 0; o >>= 1) {
        acc += __shfl_xor_sync(0xffffffffu, acc, o);
        aops += __shfl_xor_sync(0xffffffffu, aops, o);
#pragma unroll
        for (int q = 0; q < kMaxClass; ++q) items[q] += __shfl_xor_sync(0xffffffffu, items[q], o);
    }
    if ((threadIdx.x & 31) == 0 && acc) {
        atomicAdd(out, acc);
        atomicAdd(out + 1, aops);
#pragma unroll
        for (int q = 0; q < kMaxClass; ++q)
            if (items[q]) atomicAdd(out + 2 + q, items[q]);
    }
}
__global__ void tile_pair_list(const uint4* chunks, const uint32_t* nchunks, const uint32_t* jlist, uint32_t* out) {
    const unsigned n = *nchunks;
    for (unsigned c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x) {
        const uint4 ch = chunks[c];
        for (unsigned e = ch.y; e < ch.z; ++e) {
            out[2 * (size_t)e] = ch.x;
            out[2 * (size_t)e + 1] = jlist[e];
        }
    }
}
__global__ void neighbor_counts(const uint64_t* keys, long long n, long long n_cols, uint32_t* counts,
                                int64_t* flat) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const uint64_t k = keys[t];
    const uint64_t i = k / (uint64_t)n_cols;
    atomicAdd(&counts[i], 1u);
    if (flat) flat[t] = (int64_t)(k - i * (uint64_t)n_cols);
}

int bits_for(unsigned long long max_value) {
    int b = 1;
    while (b < 64 && (max_value >> b) != 0) ++b;
    return b;
}

struct Events {
    cudaEvent_t e[8];
    int n = 0;
    Events() { for (auto& x : e) cudaEventCreate(&x); }
    ~Events() { for (auto& x : e) cudaEventDestroy(x); }
    void rec(int i, cudaStream_t st) { cudaEventRecord(e[i], st); n = i + 1 > n ? i + 1 : n; }
    double ms(int a, int b) const {
        float m = 0.f;
        cudaEventElapsedTime(&m, e[a], e[b]);
        return (double)m;
    }
};

}  // namespace

// Threshold constants of the certificate.
JoinParams make_params(double T, int d, int kpad, int split, long long nr, long long nc, bool self_join) {
    JoinParams jp;
    memset(&jp, 0, sizeof(jp));
    jp.T = T;
    // |fp64 oracle value - D| <= g64 * D (d subtractions, squares and additions, u = 2^-53)
    const double nu = (double)(d + 2) * 0x1p-53;
    const double g64 = nu / (1.0 - nu);
    jp.Tm = T / (1.0 + g64) * (1.0 - 0x1p-50);
    jp.Tp = T / (1.0 - g64) * (1.0 + 0x1p-50);
    jp.gn = 2.0 * (double)(d + 2) * 0x1p-53;
    // tensor-core accumulation premise: every FP32 accumulation step of the K exact products errs by at most
    // 2 ulp of the running |sum| (2x the round-to-nearest bound, covering truncating alignment), + 64 steps slack
    const double kacc = (double)kpad * (split ? 3.0 : 1.0);
    jp.gmma = (kacc + 64.0) * 0x1p-22;
    jp.cabs = (kacc + 64.0) * 0x1p-125;
    jp.key_off = 0;
    jp.n_rows = nr;
    jp.n_cols = nc;
    jp.self_join = self_join ? 1 : 0;
    jp.d = d;
    return jp;
}

}  // namespace tj

// ====================================================================== C ABI
using namespace tj;

struct tj_result {
    DBuf<uint64_t> keys;       // sorted canonical keys (first `count` valid)
    long long count = 0;
    // TJ_FLAG_STAGE_KEYS: the screen's certified accepts (0) and its band (1), sorted, first stage_n valid
    DBuf<uint64_t> stage[2];
    long long stage_n[2] = {0, 0};
    long long n_rows = 0, n_cols = 0;
    tj_stats stats;
    // batched mode (njoins > 1): per-join output ranges and key decoding tables
    int njoins = 1;
    std::vector<int64_t> offsets;
    DBuf<unsigned long long> d_keyoff;
    DBuf<long long> d_cols;
};

struct tj_index {
    Side side;
    TileSet t128, t256;
    Candidates cand;
    DBuf<uint32_t> cell_start;
    long long n_cells = 0;
    long long n_tile_pairs = 0;
};

#define TJ_API_BEGIN try {
#define TJ_API_END                                          \
    }                                                       \
    catch (const tj::Error& e) {                            \
        g_last_error = e.msg;                               \
        return e.code;                                      \
    }                                                       \
    catch (const std::exception& e) {                       \
        g_last_error = e.what();                            \
        return TJ_ERR_INVALID;                              \
    }                                                       \
    catch (...) {                                           \
        g_last_error = "unknown error";                     \
        return TJ_ERR_INVALID;                              \
    }

namespace {

void check_status(unsigned long long status) {
    if (status & kStatusWaitTimeout) fail(TJ_ERR_TIMEOUT, "a bounded device wait expired; the kernel returned early");
    if (status & kStatusBadInput) fail(TJ_ERR_INPUT, "input contains NaN/Inf or a row norm beyond 2^50");
    if (status & kStatusFp16Range) fail(TJ_ERR_RANGE, "input magnitude exceeds the FP16 range; use the BF16 screen");
    if (status & kStatusTmemAlloc) fail(TJ_ERR_CUDA, "tensor memory allocation failed");
    if (status & kStatusGuard) fail(TJ_ERR_CUDA, "a guard region after an output buffer was overwritten");
}

struct JoinIn {
    const void* R;
    const void* S;
    long long nR, nS;
    int d;
    double eps2;
};

void check_flags(const tj_options* opt) {
    if (!opt) return;
    const int known = TJ_FLAG_SCREEN_DIAG | TJ_FLAG_SCREEN_1SM | TJ_FLAG_FRAME_AXES | TJ_FLAG_FRAME_PCA |
                      TJ_FLAG_BAND_FP32 | TJ_FLAG_I8_FOUR_PRODUCTS | TJ_FLAG_GUARDS | TJ_FLAG_STAGE_KEYS |
                      TJ_FLAG_SCREEN_TIMES | TJ_FLAG_WHOLE_TILES;
    if (opt->flags & ~known) fail(TJ_ERR_INVALID, "unknown option flags");
    if ((opt->flags & TJ_FLAG_FRAME_AXES) && (opt->flags & TJ_FLAG_FRAME_PCA))
        fail(TJ_ERR_INVALID, "TJ_FLAG_FRAME_AXES and TJ_FLAG_FRAME_PCA exclude each other");
    if (opt->k_block != 0 && opt->k_block != 16 && opt->k_block != 32 && opt->k_block != 64)
        fail(TJ_ERR_INVALID, "k_block must be 0, 16, 32 or 64");
    if (opt->stages != 0 && (opt->stages < 2 || opt->stages > 6)) fail(TJ_ERR_INVALID, "stages must be 0 or 2..6");
}

// One or many joins.  Joins are grouped into classes of equal d; each class gets one
// concatenated, Morton-sorted side per operand (joins stay contiguous), global tile tables, one
// block-diagonal candidate list and one persistent screen launch over all classes.
void run_batch_body(const std::vector<JoinIn>& joins, int dtype, int mode, int screen, const tj_options* opt,
                    tj_result* res, cudaStream_t st) {
    const bool self = mode != TJ_MODE_RS;
    const int nj = (int)joins.size();
    if (nj < 1) fail(TJ_ERR_INVALID, "no joins");
    if (self && nj != 1) fail(TJ_ERR_INVALID, "self-join modes take one join");
    const bool i8 = screen == TJ_SCREEN_INT8LIMB;
    if (i8 && nj != 1) fail(TJ_ERR_UNSUPPORTED, "the int8-limb screen runs one join at a time");
    if (dtype == TJ_DTYPE_I16 && !i8) fail(TJ_ERR_UNSUPPORTED, "int16 input needs the int8-limb screen");
    if (dtype == TJ_DTYPE_F32 && i8) fail(TJ_ERR_UNSUPPORTED, "the int8-limb screen needs int16 (int14) input");
    long long total_r = 0;
    for (const auto& j : joins) {
        if ((j.nR > 0 && !j.R) || (j.nS > 0 && !j.S)) fail(TJ_ERR_INVALID, "null input pointer");
        if (j.d <= 0 || j.nR < 0 || j.nS < 0) fail(TJ_ERR_INVALID, "invalid shape");
        if (j.nR >= (1ll << 32) || j.nS >= (1ll << 32)) fail(TJ_ERR_INVALID, "more than 2^32 - 1 rows per side");
        if (!(j.eps2 >= 0.0) || std::isinf(j.eps2)) fail(TJ_ERR_INVALID, "eps2 must be finite and >= 0");
        if (i8 && !(j.eps2 == std::floor(j.eps2) && j.eps2 < 0x1p62))
            fail(TJ_ERR_INVALID, "the int8-limb screen needs an integer eps2 below 2^62");
        total_r += j.nR;
    }
    const int chunk_items = (opt && opt->chunk_items > 0) ? opt->chunk_items : 64;
    const int esize = dtype == TJ_DTYPE_I16 ? 2 : 4;
    tj_stats& S_ = res->stats;
    memset(&S_, 0, sizeof(S_));
    res->njoins = nj;
    res->n_rows = nj == 1 ? joins[0].nR : total_r;
    res->n_cols = nj == 1 ? (self ? joins[0].nR : joins[0].nS) : 0;
    S_.n_rows = res->n_rows;
    S_.n_cols = res->n_cols;

    // key space: join k owns [key_off[k], key_off[k] + nR_k * nS_k)
    std::vector<unsigned long long> key_off(nj);
    std::vector<long long> ncols(nj);
    unsigned long long kspace = 0;
    for (int k = 0; k < nj; ++k) {
        const long long nc = self ? joins[k].nR : joins[k].nS;
        key_off[k] = kspace;
        ncols[k] = nc;
        kspace += (unsigned long long)joins[k].nR * (unsigned long long)nc;
        S_.pairs_all += self ? joins[k].nR * (joins[k].nR - 1) / 2 : joins[k].nR * joins[k].nS;
    }
    // classes of equal d (joins with an empty side contribute no pairs and are skipped)
    std::vector<int> cls_d;
    std::vector<std::vector<int>> cls_j;
    for (int k = 0; k < nj; ++k) {
        if (joins[k].nR == 0 || (!self && joins[k].nS == 0)) continue;
        int c = -1;
        for (size_t q = 0; q < cls_d.size(); ++q)
            if (cls_d[q] == joins[k].d) c = (int)q;
        if (c < 0) {
            if ((int)cls_d.size() == kMaxClass) fail(TJ_ERR_UNSUPPORTED, "at most 4 distinct dimensions per batch");
            cls_d.push_back(joins[k].d);
            cls_j.emplace_back();
            c = (int)cls_d.size() - 1;
        }
        cls_j[c].push_back(k);
    }
    const int ncls = (int)cls_d.size();
    if (ncls == 0) {
        res->count = 0;
        if (nj > 1) res->offsets.assign(nj + 1, 0);
        return;
    }
    stage_reset();
    Events ev;
    ev.rec(0, st);
    DBuf<Counters> ctr(1, st);
    launch(zero_counters, 1, 32, 0, st, ctr.p, 0);

    struct Cls {
        Side R, S;
        TileSet tR, tS;
        TileSet tSh;   // 128-row halves of the S tiles (half-tile masks of the one-SM screen)
        DBuf<float> XR, XS, center;
        DBuf<FrameParams> fp;
        bool pca_frame = false;   // cells over principal directions (else input dimensions)
        DBuf<long long> rowoffR, rowoffS;
    };
    std::vector<std::unique_ptr<Cls>> C(ncls);
    std::vector<uint4> rtiles, stiles;
    ScreenInput g;
    g.ncls = ncls;
    std::vector<JoinParams> jps(nj);
    for (int k = 0; k < nj; ++k) memset(&jps[k], 0, sizeof(JoinParams));
    const int stile = i8 ? 128 : kTileS;
    // live 128-row halves of every candidate for the one-SM 16-bit screen (joins the CTA-pair screen
    // is likely to take skip this: that screen walks the whole tile grid; such joins have rows of
    // more than 192 elements, kpad >= 256, and no hi/lo split)
    const bool tc16 = !i8 && screen != TJ_SCREEN_PLAIN;
    const bool split_screen = screen == TJ_SCREEN_BF16X3 || screen == TJ_SCREEN_FP16X3;
    const bool allow_pair = !(opt && (opt->flags & TJ_FLAG_SCREEN_1SM));
    const bool likely_pair = allow_pair && ncls == 1 && nj == 1 && !self && !split_screen && cls_d[0] > 192;
    const bool diag_req = opt && (opt->flags & TJ_FLAG_SCREEN_DIAG) && tc16;   // samples whole tile pairs
    // (the half-tile test keeps eight R tiles' centroid and box in shared memory: rows of at most
    // 2048 elements)
    const bool half_packed = tc16 && !likely_pair && !diag_req && !(opt && (opt->flags & TJ_FLAG_WHOLE_TILES)) &&
                             *std::max_element(cls_d.begin(), cls_d.end()) <= 2048;
    for (int c = 0; c < ncls; ++c) {
        C[c].reset(new Cls());
        Cls& K = *C[c];
        const int d = cls_d[c];
        const auto& J = cls_j[c];
        const int njc = (int)J.size();
        std::vector<long long> roR(njc + 1, 0), roS(njc + 1, 0);
        for (int q = 0; q < njc; ++q) {
            roR[q + 1] = roR[q] + joins[J[q]].nR;
            roS[q + 1] = roS[q] + (self ? joins[J[q]].nR : joins[J[q]].nS);
        }
        const void* srcR = joins[J[0]].R;
        const void* srcS = self ? joins[J[0]].R : joins[J[0]].S;
        if (njc > 1) {   // concatenate the class's joins (one copy per side)
            std::vector<const void*> pr, ps;
            std::vector<long long> nr, ns;
            for (int q = 0; q < njc; ++q) {
                pr.push_back(joins[J[q]].R); nr.push_back(joins[J[q]].nR);
                ps.push_back(joins[J[q]].S); ns.push_back(joins[J[q]].nS);
            }
            // joins whose rows already lie back to back in one array (views of one tensor) are used
            // in place; otherwise the class's rows are gathered into one array
            auto adjacent = [&](const std::vector<const void*>& p, const std::vector<long long>& n) {
                for (size_t q = 0; q + 1 < p.size(); ++q)
                    if ((const char*)p[q] + (size_t)n[q] * d * esize != (const char*)p[q + 1]) return false;
                return true;
            };
            if (adjacent(pr, nr)) {
                srcR = pr[0];
            } else {
                K.XR = DBuf<float>((size_t)roR[njc] * d, st);
                gather_rows(pr, nr, d, esize, K.XR.p, st);
                srcR = K.XR.p;
            }
            if (self) {
                srcS = srcR;
            } else if (adjacent(ps, ns)) {
                srcS = ps[0];
            } else {
                K.XS = DBuf<float>((size_t)roS[njc] * d, st);
                gather_rows(ps, ns, d, esize, K.XS.p, st);
                srcS = K.XS.p;
            }
            K.rowoffR = DBuf<long long>((size_t)njc + 1, st);
            K.rowoffS = DBuf<long long>((size_t)njc + 1, st);
            upload(K.rowoffR.p, roR.data(), (njc + 1) * 8, st);
            upload(K.rowoffS.p, roS.data(), (njc + 1) * 8, st);
        }
        K.fp = DBuf<FrameParams>(1, st);
        K.center = DBuf<float>((size_t)d, st);
        {
            const void* srcs[2] = {srcR, srcS};
            const long long ns[2] = {roR[njc], roS[njc]};
            // packed joins keep input-dimension cells unless asked otherwise: one covariance pooled
            // over many joins mostly describes how the joins differ, not how each one's rows spread
            const int flags = opt ? opt->flags : 0;
            const int fm = (flags & TJ_FLAG_FRAME_AXES) ? kFrameAxes
                         : (flags & TJ_FLAG_FRAME_PCA) ? kFramePca
                         : njc == 1 ? kFrameAuto : kFrameAxes;
            K.pca_frame = compute_frame(srcs, ns, self ? 1 : 2, d, dtype, fm, K.fp.p, K.center.p, st);
            if (K.pca_frame) S_.index_frame = 1;
        }
        // tile tables: tiles never span two joins; sorted rows of join q are [ro[q], ro[q+1])
        g.rbase[c] = (int)rtiles.size();
        g.sbase[c] = (int)stiles.size();
        {
            size_t ntr = 0, nts = 0;
            for (int q = 0; q < njc; ++q) {
                const int k = J[q];
                ntr += (size_t)((joins[k].nR + kTileR - 1) / kTileR);
                nts += (size_t)(((self ? joins[k].nR : joins[k].nS) + stile - 1) / stile);
            }
            for (auto* v : {&K.tR.h_row0, &K.tR.h_nvalid, &K.tR.h_join}) v->reserve(ntr);
            for (auto* v : {&K.tS.h_row0, &K.tS.h_nvalid, &K.tS.h_join}) v->reserve(nts);
            rtiles.reserve(rtiles.size() + ntr);
            stiles.reserve(stiles.size() + nts);
        }
        for (int q = 0; q < njc; ++q) {
            const int k = J[q];
            for (long long t = 0; t * kTileR < joins[k].nR; ++t) {
                const uint32_t r0 = (uint32_t)(roR[q] + t * kTileR);
                const uint32_t nv = (uint32_t)std::min<long long>(kTileR, joins[k].nR - t * kTileR);
                K.tR.h_row0.push_back(r0); K.tR.h_nvalid.push_back(nv); K.tR.h_join.push_back((uint32_t)k);
                rtiles.push_back(make_uint4(r0, nv, (unsigned)k, (unsigned)c));
            }
            const long long nsk = self ? joins[k].nR : joins[k].nS;
            for (long long t = 0; t * stile < nsk; ++t) {
                const uint32_t r0 = (uint32_t)(roS[q] + t * stile);
                const uint32_t nv = (uint32_t)std::min<long long>(stile, nsk - t * stile);
                K.tS.h_row0.push_back(r0); K.tS.h_nvalid.push_back(nv); K.tS.h_join.push_back((uint32_t)k);
                stiles.push_back(make_uint4(r0, nv, (unsigned)k, (unsigned)c));
            }
        }
        // operands and tile statistics (one fused pass per side where the side allows it: the R
        // tiling, or for a self-join the S tiling; the S tiling brings its 128-row halves along when
        // the screen packs half-tiles)
        TileSet* halves = half_packed ? &K.tSh : nullptr;
        K.R.src = srcR; K.R.dtype = dtype; K.R.n = roR[njc]; K.R.d = d; K.R.screen = screen;
        K.R.njc = njc; K.R.d_rowoff = njc > 1 ? K.rowoffR.p : nullptr;
        if (self)
            prepare_side(K.R, K.fp.p, K.pca_frame, K.center.p, st, &ctr.p->status, &K.tS, stile, halves);
        else
            prepare_side(K.R, K.fp.p, K.pca_frame, K.center.p, st, &ctr.p->status, &K.tR, kTileR);
        compute_perm_local(K.R, st);
        Side* pS = &K.R;
        if (!self) {
            K.S.src = srcS; K.S.dtype = dtype; K.S.n = roS[njc]; K.S.d = d; K.S.screen = screen;
            K.S.njc = njc; K.S.d_rowoff = njc > 1 ? K.rowoffS.p : nullptr;
            prepare_side(K.S, K.fp.p, K.pca_frame, K.center.p, st, &ctr.p->status, &K.tS, stile, halves);
            compute_perm_local(K.S, st);
            pS = &K.S;
        }
        tile_stats(K.R, kTileR, K.tR, st);
        tile_stats(*pS, stile, K.tS, st);
        for (int q = 0; q < njc; ++q) {
            const int k = J[q];
            jps[k] = make_params(joins[k].eps2, d, K.R.kpad, K.R.split, joins[k].nR, ncols[k], self);
            jps[k].key_off = key_off[k];
        }
        g.R[c] = &K.R;
        g.S[c] = pS;
        g.tR[c] = &K.tR;
        g.tS[c] = &K.tS;
    }
    g.ntR_total = (int)rtiles.size();
    g.ntS_total = (int)stiles.size();
    g.njoins = nj;
    g.jp0 = jps[0];
    g.T_int = (long long)joins[0].eps2;
    DBuf<uint4> d_rt((size_t)g.ntR_total, st), d_st((size_t)g.ntS_total, st);
    DBuf<JoinParams> d_jps((size_t)nj, st);
    DBuf<unsigned long long> d_koff;
    DBuf<long long> d_cols;
    {
        WorkspaceSuspend keep;   // key decoding tables stay with the result
        d_koff = DBuf<unsigned long long>((size_t)nj, st);
        d_cols = DBuf<long long>((size_t)nj, st);
    }
    DBuf<const void*> d_rsrc((size_t)nj, st), d_ssrc((size_t)nj, st);
    std::vector<const void*> hr(nj), hs(nj);
    for (int k = 0; k < nj; ++k) { hr[k] = joins[k].R; hs[k] = self ? joins[k].R : joins[k].S; }
    upload(d_rt.p, rtiles.data(), rtiles.size() * sizeof(uint4), st);
    upload(d_st.p, stiles.data(), stiles.size() * sizeof(uint4), st);
    upload(d_jps.p, jps.data(), nj * sizeof(JoinParams), st);
    upload(d_koff.p, key_off.data(), nj * 8, st);
    upload(d_cols.p, ncols.data(), nj * 8, st);
    upload(d_rsrc.p, hr.data(), nj * sizeof(void*), st);
    upload(d_ssrc.p, hs.data(), nj * sizeof(void*), st);
    g.rtiles = d_rt.p;
    g.stiles = d_st.p;
    g.jps = d_jps.p;
    g.h_jps = jps.data();
    g.allow_pair = allow_pair;
    g.i8_four_products = opt && (opt->flags & TJ_FLAG_I8_FOUR_PRODUCTS);
    g.k_block = opt ? opt->k_block : 0;
    g.stages = opt ? opt->stages : 0;
    g.key_off = d_koff.p;
    g.rsrc = d_rsrc.p;
    g.ssrc = d_ssrc.p;
    ev.rec(1, st);

    // candidate tile pairs (block-diagonal over joins) and execution chunks
    Candidates cand;
    if (nj == 1) {
        build_candidates(*g.tR[0], *g.tS[0], jps[0].Tp, self, chunk_items, cand, st);
    } else {
        std::vector<CandClassView> views(ncls);
        for (int c = 0; c < ncls; ++c) {
            const TileSet& a = *g.tR[c];
            const TileSet& b = *g.tS[c];
            views[c] = CandClassView{a.ctrT.p, a.loT.p, a.hiT.p, a.rad.p, b.ctrT.p, b.loT.p, b.hiT.p, b.rad.p,
                                     a.ntiles, b.ntiles, g.rbase[c], g.sbase[c], cls_d[c], 0};
        }
        std::vector<CandBlock> blocks;
        std::vector<double> tps;
        std::vector<uint32_t> rsb(g.ntR_total, 0);
        int words = 1;
        std::vector<int> jr0(nj, -1), js0(nj, -1), jnr(nj, 0), jns(nj, 0), jcls(nj, 0);
        for (int i = 0; i < g.ntR_total; ++i) {
            const int k = (int)rtiles[i].z;
            if (jr0[k] < 0) jr0[k] = i;
            ++jnr[k];
            jcls[k] = (int)rtiles[i].w;
        }
        for (int i = 0; i < g.ntS_total; ++i) {
            const int k = (int)stiles[i].z;
            if (js0[k] < 0) js0[k] = i;
            ++jns[k];
        }
        for (int k = 0; k < nj; ++k) {
            if (jr0[k] < 0 || js0[k] < 0) continue;
            words = std::max(words, (jns[k] + 31) / 32);
            for (int t = 0; t < jnr[k]; t += 16) {
                blocks.push_back(CandBlock{(uint32_t)(jr0[k] + t), (uint32_t)std::min(16, jnr[k] - t),
                                           (uint32_t)js0[k], (uint32_t)jns[k], (uint32_t)jcls[k], 0u});
                tps.push_back(jps[k].Tp);
            }
            for (int t = 0; t < jnr[k]; ++t) rsb[jr0[k] + t] = (uint32_t)js0[k];
        }
        build_candidates_batched(views, blocks, tps, g.ntR_total, words, chunk_items, rsb, cand, st);
    }
    g.cand = &cand;
    ScreenOps sops;
    memset(&sops, 0, sizeof(sops));
    for (int c = 0; c < ncls; ++c) {
        sops.per_pair[c] = (unsigned long long)cls_d[c] * (i8 ? 8ull : (C[c]->R.split ? 6ull : 2ull));
        // one half-item issues 2 M N K per product: 128 x 128 (16-bit, 3 products with the split; a
        // tile pair is two half-items) or 128 x 128 x 1/2 (int8: an item is one 128 x 128 tile pair,
        // counted as two halves, of which the high-limb screen issues hh only)
        sops.per_item[c] = 2.0 * kTileR * 128.0 * (double)C[c]->R.kpad * (C[c]->R.split ? 3.0 : 1.0) *
                           (i8 ? 0.5 : 1.0);
    }
    g.half_packed = half_packed;
    if (g.half_packed) {
        std::vector<HalfView> hv(ncls);
        for (int c = 0; c < ncls; ++c) {
            Cls& K = *C[c];
            TileSet& H = K.tSh;
            if (!H.built) {   // halves not made by the fused operand pass
                for (size_t t = 0; t < K.tS.h_row0.size(); ++t)
                    for (uint32_t h = 0; h < 2; ++h) {
                        const uint32_t nv = K.tS.h_nvalid[t];
                        H.h_row0.push_back(K.tS.h_row0[t] + 128u * h);
                        H.h_nvalid.push_back(nv > 128u * h ? std::min(128u, nv - 128u * h) : 0u);
                    }
                tile_stats(*g.S[c], 128, H, st);
            }
            tile_stats_rowmajor(H, st);
            hv[c] = HalfView{K.tR.ctrT.p, K.tR.loT.p, K.tR.hiT.p, K.tR.rad.p, H.ctrR.p, H.loR.p, H.hiR.p, H.rad.p,
                             H.nvalid.p, K.tR.ntiles, H.ntiles, g.rbase[c], g.sbase[c], cls_d[c], 0};
        }
        half_masks(hv, cand, g.ntR_total, d_rt.p, d_jps.p, self, st);
    }
    launch(pairs_screened_kernel, num_sms() * 4, 256, 0, st, (const uint4*)cand.chunks.p,
           (const uint32_t*)(cand.dev_counts.p + 1), (const uint32_t*)cand.jlist.p, (const uint4*)d_rt.p,
           (const uint4*)d_st.p, sops, g.half_packed ? 1 : 0, &ctr.p->pairs_screened);
    ev.rec(6, st);

    // optional screen-error sampling (tensor-core screens): 64 tile pairs spread over the candidate list
    const bool diag = opt && (opt->flags & TJ_FLAG_SCREEN_DIAG) && screen != TJ_SCREEN_PLAIN && !i8;
    const bool band_fp32 = opt && (opt->flags & TJ_FLAG_BAND_FP32);
    DBuf<float> dump;
    DBuf<uint4> dump_ids;
    DBuf<unsigned long long> diag_out;
    if (diag) {
        uint32_t tot = 0;
        TJ_CUDA(cudaMemcpyAsync(&tot, cand.dev_counts.p, 4, cudaMemcpyDeviceToHost, st));
        TJ_CUDA(cudaStreamSynchronize(st));
        g.dump_items = 64;
        g.dump_every = std::max(1u, tot / g.dump_items);
        dump = DBuf<float>((size_t)g.dump_items * kTileR * kTileS, st);
        dump_ids = DBuf<uint4>(g.dump_items, st);
        diag_out = DBuf<unsigned long long>(3, st);
        TJ_CUDA(cudaMemsetAsync(dump_ids.p, 0, g.dump_items * sizeof(uint4), st));
        TJ_CUDA(cudaMemsetAsync(diag_out.p, 0, 3 * 8, st));
        g.dump = dump.p;
        g.dump_ids = dump_ids.p;
        g.diag_out = diag_out.p;
    }

    // screen + refine with overflow-and-retry
    unsigned long long sum_max = 0;
    for (const auto& j : joins) sum_max += (unsigned long long)std::max(j.nR, self ? j.nR : j.nS);
    const unsigned long long per = nj == 1 ? 64ull : 24ull;
    unsigned long long cap = (opt && opt->initial_capacity > 0) ? (unsigned long long)opt->initial_capacity
                                                                : std::max<unsigned long long>(1ull << 20, per * sum_max);
    unsigned long long bcap = (opt && opt->initial_capacity > 0) ? cap : std::max<unsigned long long>(1ull << 20,
                                                                                                   cap / (nj == 1 ? 1 : 8));
    const bool guards = opt && (opt->flags & TJ_FLAG_GUARDS);
    const bool stage_keys = opt && (opt->flags & TJ_FLAG_STAGE_KEYS);
    const unsigned long long gs = guards ? kGuardSlots : 0;
    const bool times = opt && (opt->flags & TJ_FLAG_SCREEN_TIMES) && screen != TJ_SCREEN_PLAIN && !i8;
    DBuf<unsigned long long> join_t, cta_t, role_t;
    if (times) {
        join_t = DBuf<unsigned long long>(2 * (size_t)nj, st);
        cta_t = DBuf<unsigned long long>(2 * (size_t)num_sms(), st);
        role_t = DBuf<unsigned long long>(16, st);
        g.join_t = join_t.p;
        g.cta_t = cta_t.p;
        g.role_t = role_t.p;
    }
    DBuf<uint64_t> acc, band;
    Counters h;
    for (int attempt = 0;; ++attempt) {
        acc = DBuf<uint64_t>::result(cap + gs, st);   // becomes the result's key array
        band = DBuf<uint64_t>(bcap + gs, st);
        launch(zero_counters, 1, 32, 0, st, ctr.p, 1);
        if (times) {   // first starts: all ones (atomicMin), last ends and CTA stamps: zero
            TJ_CUDA(cudaMemsetAsync(join_t.p, 0xFF, (size_t)nj * 8, st));
            TJ_CUDA(cudaMemsetAsync(join_t.p + nj, 0, (size_t)nj * 8, st));
            TJ_CUDA(cudaMemsetAsync(cta_t.p, 0, cta_t.bytes(), st));
            TJ_CUDA(cudaMemsetAsync(role_t.p, 0, role_t.bytes(), st));
        }
        if (guards) {
            launch(guard_fill, 1, 256, 0, st, acc.p + cap);
            launch(guard_fill, 1, 256, 0, st, band.p + bcap);
        }
        EmitBuffers eb{acc.p, cap, band.p, bcap, ctr.p};
        ev.rec(2, st);
        if (screen == TJ_SCREEN_PLAIN) screen_plain(g, eb, st);
        else if (i8) screen_i8(g, eb, st);
        else screen_tc(g, eb, st);
        S_.screen_pair = g.used_pair ? 1 : 0;
        ev.rec(3, st);
        if (stage_keys) launch(snapshot_reserved, 1, 1, 0, st, ctr.p);
        // the four-product int8-limb screen is exact: no band; the plain screen's band is already the
        // FP32 stage's undecided set
        if (!i8 || i8_high_limb_screen(g)) refine_band(g, eb, band_fp32 && screen != TJ_SCREEN_PLAIN && !i8, st);
        ev.rec(4, st);
        if (guards) {
            launch(guard_check, 1, 256, 0, st, (const uint64_t*)(acc.p + cap), ctr.p);
            launch(guard_check, 1, 256, 0, st, (const uint64_t*)(band.p + bcap), ctr.p);
        }
        TJ_CUDA(cudaMemcpyAsync(&h, ctr.p, sizeof(Counters), cudaMemcpyDeviceToHost, st));
        TJ_CUDA(cudaStreamSynchronize(st));
        check_status(h.status);
        const bool over = h.acc_reserved > cap || h.band_reserved > bcap;
        if (!over) break;
        if (attempt >= 6) fail(TJ_ERR_NOMEM, "output capacity retries exhausted");
        S_.retries++;
        cap = std::max(cap * 2, h.acc_reserved + h.acc_reserved / 4 + 4096);
        bcap = std::max(bcap * 2, h.band_reserved + h.band_reserved / 4 + 4096);
    }
    S_.tile_pairs = (int64_t)h.items;
    S_.pairs_screened = (int64_t)h.pairs_screened;
    S_.screen_ops = (double)h.screen_ops;
    for (int c = 0; c < ncls; ++c) S_.screen_ops_issued += (double)h.class_items[c] * sops.per_item[c];
    if (i8 && !i8_high_limb_screen(g))   // the four-product screen: hl + lh and ll for the items that took them
        S_.screen_ops_issued += 3.0 * (double)h.xl_items * 2.0 * kTileR * 128.0 * (double)C[0]->R.kpad;
    if (diag) {
        unsigned long long dv[3] = {0, 0, 0};
        TJ_CUDA(cudaMemcpyAsync(dv, diag_out.p, sizeof(dv), cudaMemcpyDeviceToHost, st));
        TJ_CUDA(cudaStreamSynchronize(st));
        memcpy(&S_.screen_max_abs_err, &dv[0], 8);
        memcpy(&S_.screen_err_over_bound, &dv[1], 8);
        S_.screen_err_pairs = (int64_t)dv[2];
    }
    if (times) {
        std::vector<unsigned long long> jt(2 * (size_t)nj), ct(cta_t.n), rl(16);
        TJ_CUDA(cudaMemcpyAsync(jt.data(), join_t.p, jt.size() * 8, cudaMemcpyDeviceToHost, st));
        TJ_CUDA(cudaMemcpyAsync(ct.data(), cta_t.p, ct.size() * 8, cudaMemcpyDeviceToHost, st));
        TJ_CUDA(cudaMemcpyAsync(rl.data(), role_t.p, rl.size() * 8, cudaMemcpyDeviceToHost, st));
        TJ_CUDA(cudaStreamSynchronize(st));
        std::vector<double> span;
        for (int k = 0; k < nj; ++k)
            if (jt[nj + k] && jt[k] != ~0ull && jt[nj + k] >= jt[k]) span.push_back((double)(jt[nj + k] - jt[k]) * 1e-6);
        std::sort(span.begin(), span.end());
        if (!span.empty()) {
            auto pct = [&](double p) { return span[std::min(span.size() - 1, (size_t)(p * (double)(span.size() - 1) + 0.5))]; };
            S_.join_span_ms_p50 = pct(0.5);
            S_.join_span_ms_p99 = pct(0.99);
            S_.join_span_ms_max = span.back();
        }
        unsigned long long lo = ~0ull, hi = 0;
        for (size_t b = 0; b + 1 < ct.size(); b += 2)
            if (ct[b + 1]) { lo = std::min(lo, ct[b + 1]); hi = std::max(hi, ct[b + 1]); }
        if (hi >= lo && hi) S_.screen_cta_tail_ms = (double)(hi - lo) * 1e-6;
        // stall accounting: slots as the screen's RoleSlot (producer 0-2, issuer 3-5, epilogue 6-11)
        auto frac = [&](int part, int whole) { return rl[whole] ? (double)rl[part] / (double)rl[whole] : 0.0; };
        S_.screen_prod_stage_wait = frac(1, 0);
        S_.screen_prod_meta_wait = frac(2, 0);
        S_.screen_mma_operand_wait = frac(4, 3);
        S_.screen_mma_acc_wait = frac(5, 3);
        S_.screen_epi_meta_wait = frac(7, 6);
        S_.screen_epi_acc_wait = frac(8, 6);
        S_.screen_epi_test = frac(9, 6);
        S_.screen_epi_emit = frac(10, 6);
        S_.screen_epi_reserve = frac(11, 6);
    }
    S_.screen_accept = (int64_t)h.screen_accept;
    S_.band = (int64_t)h.band_valid;
    S_.refine_accept = (int64_t)h.refine_accept;
    S_.rare_checks = (int64_t)h.rare_checks;
    S_.band_fp64 = (int64_t)h.band_fp64;
    if (stage_keys) {   // the screen's own decisions, sorted (self-joins: the screen's i < j form)
        WorkspaceSuspend keep;
        const unsigned long long n0 = std::min(h.screen_reserved, cap), n1 = std::min(h.band_reserved, bcap);
        const uint64_t* src[2] = {acc.p, band.p};
        const unsigned long long ns[2] = {n0, n1};
        res->stage_n[0] = (long long)h.screen_accept;
        res->stage_n[1] = (long long)h.band_valid;
        for (int q = 0; q < 2; ++q) {
            res->stage[q] = DBuf<uint64_t>(std::max(ns[q], 1ull), st);
            if (!ns[q]) continue;
            TJ_CUDA(cudaMemcpyAsync(res->stage[q].p, src[q], ns[q] * 8, cudaMemcpyDeviceToDevice, st));
            if (ns[q] > 1) {
                DBuf<uint64_t> t(ns[q], st);
                DBuf<uint32_t> w(radix_workspace_elems(ns[q]), st);
                radix_sort(res->stage[q].p, nullptr, t.p, nullptr, ns[q], 64, w.p, st, &ctr.p->status);
            }
        }
    }
    band.reset();

    // canonical order
    unsigned long long slots = h.acc_reserved;
    long long nvalid = (long long)h.acc_valid;
    DBuf<uint64_t> keys;
    if (mode == TJ_MODE_DIRECTED) {
        const long long N = joins[0].nR;
        const unsigned long long nk = 2 * slots + (unsigned long long)N;
        keys = DBuf<uint64_t>::result(nk + gs, st);
        expand_directed(acc.p, slots, keys.p, N, st);
        acc.reset();
        slots = nk;
        nvalid = 2 * nvalid + N;
    } else {
        keys = std::move(acc);
    }
    const int bits = bits_for(kspace);   // sentinel low bits (all ones) exceed every valid key
    if (guards) launch(guard_fill, 1, 256, 0, st, keys.p + slots);   // keys holds >= slots + gs words
    if (slots > 1) {
        // an odd number of single-sweep passes ends in the temporaries: they are then a result buffer
        // and the two buffers change places instead of copying the keys back
        const bool swap = radix_result_in_tmp(slots, bits);
        DBuf<uint64_t> ktmp = swap ? DBuf<uint64_t>::result(slots + gs, st) : DBuf<uint64_t>(slots + gs, st);
        DBuf<uint32_t> ws(radix_workspace_elems(slots), st);
        if (guards) launch(guard_fill, 1, 256, 0, st, ktmp.p + slots);
        bool in_tmp = false;
        radix_sort(keys.p, nullptr, ktmp.p, nullptr, slots, bits, ws.p, st, &ctr.p->status, swap ? &in_tmp : nullptr);
        if (guards) launch(guard_check, 1, 256, 0, st, (const uint64_t*)(ktmp.p + slots), ctr.p);
        if (in_tmp) std::swap(keys, ktmp);
    }
    if (guards) launch(guard_check, 1, 256, 0, st, (const uint64_t*)(keys.p + slots), ctr.p);
    if (nj > 1) {
        DBuf<long long> offs((size_t)nj + 1, st);
        batch_offsets(keys.p, nvalid, d_koff.p, nj, offs.p, st);
        res->offsets.resize(nj + 1);
        TJ_CUDA(cudaMemcpyAsync(res->offsets.data(), offs.p, (nj + 1) * 8, cudaMemcpyDeviceToHost, st));
        res->d_keyoff = std::move(d_koff);
        res->d_cols = std::move(d_cols);
    }
    ev.rec(5, st);
    unsigned long long status_after = 0;
    if (guards)
        TJ_CUDA(cudaMemcpyAsync(&status_after, &ctr.p->status, 8, cudaMemcpyDeviceToHost, st));
    TJ_CUDA(cudaStreamSynchronize(st));
    check_status(status_after);
    res->keys = std::move(keys);
    res->count = nvalid;
    S_.result_pairs = nvalid;
    S_.ms_index = ev.ms(0, 1);
    S_.ms_candidates = ev.ms(1, 6);
    S_.ms_screen = ev.ms(2, 3);
    S_.ms_refine = ev.ms(3, 4);
    S_.ms_sort = ev.ms(4, 5);
    S_.ms_total = ev.ms(0, 5);
}

// One join (or batch) with its temporaries in the calling thread's workspace.
void run_batch(const std::vector<JoinIn>& joins, int dtype, int mode, int screen, const tj_options* opt,
               tj_result* res, cudaStream_t st) {
    WorkspaceScope ws(st);
    run_batch_body(joins, dtype, mode, screen, opt, res, st);
}

}  // namespace

extern "C" {

int tj_join(const void* R, int64_t nR, const void* S, int64_t nS, int32_t d, int32_t dtype, double eps2,
            int32_t mode, int32_t screen, const tj_options* opt, tj_result** out, void* stream) {
    TJ_API_BEGIN
    if (!out) fail(TJ_ERR_INVALID, "out is null");
    *out = nullptr;
    if (mode < 0 || mode > 2) fail(TJ_ERR_INVALID, "unknown mode");
    if (screen < 0 || screen > 5) fail(TJ_ERR_INVALID, "unknown screen");
    if (dtype != TJ_DTYPE_F32 && dtype != TJ_DTYPE_I16) fail(TJ_ERR_INVALID, "unknown dtype");
    check_flags(opt);
    std::unique_ptr<tj_result> res(new tj_result());
    std::vector<JoinIn> js{JoinIn{R, (const void*)(mode == TJ_MODE_RS ? S : R), nR, mode == TJ_MODE_RS ? nS : nR,
                                  d, eps2}};
    run_batch(js, dtype, mode, screen, opt, res.get(), (cudaStream_t)stream);
    *out = res.release();
    return TJ_OK;
    TJ_API_END
}

int64_t tj_result_count(const tj_result* res) { return res ? res->count : -1; }

int tj_result_stats(const tj_result* res, tj_stats* out) {
    if (!res || !out) { g_last_error = "null argument"; return TJ_ERR_INVALID; }
    *out = res->stats;
    return TJ_OK;
}

int tj_result_pairs(const tj_result* res, int64_t* i_out, int64_t* j_out, void* stream) {
    TJ_API_BEGIN
    if (!res) fail(TJ_ERR_INVALID, "null result");
    if (res->count == 0) return TJ_OK;
    if (!i_out || !j_out) fail(TJ_ERR_INVALID, "null output");
    if (res->njoins > 1) fail(TJ_ERR_INVALID, "batched result: use tj_batch_pairs");
    decode_pairs(res->keys.p, res->count, res->n_cols, i_out, j_out, (cudaStream_t)stream);
    return TJ_OK;
    TJ_API_END
}

int tj_result_keys(const tj_result* res, uint64_t* keys_out, void* stream) {
    TJ_API_BEGIN
    if (!res) fail(TJ_ERR_INVALID, "null result");
    if (res->count == 0) return TJ_OK;
    if (!keys_out) fail(TJ_ERR_INVALID, "null output");
    TJ_CUDA(cudaMemcpyAsync(keys_out, res->keys.p, (size_t)res->count * 8, cudaMemcpyDeviceToDevice,
                            (cudaStream_t)stream));
    return TJ_OK;
    TJ_API_END
}

int tj_result_stage_keys(const tj_result* res, int32_t stage, uint64_t* keys_out, int64_t* count, void* stream) {
    TJ_API_BEGIN
    if (!res || !count) fail(TJ_ERR_INVALID, "null argument");
    if (stage != 0 && stage != 1) fail(TJ_ERR_INVALID, "stage must be 0 (screen accepts) or 1 (band)");
    if (!res->stage[stage].p) fail(TJ_ERR_INVALID, "the join did not keep its stage keys (TJ_FLAG_STAGE_KEYS)");
    *count = res->stage_n[stage];
    if (keys_out && res->stage_n[stage] > 0)
        TJ_CUDA(cudaMemcpyAsync(keys_out, res->stage[stage].p, (size_t)res->stage_n[stage] * 8,
                                cudaMemcpyDeviceToDevice, (cudaStream_t)stream));
    return TJ_OK;
    TJ_API_END
}

int tj_result_neighbor_table(const tj_result* res, uint32_t* counts_out, int64_t* flat_out, void* stream) {
    TJ_API_BEGIN
    if (!res || !counts_out) fail(TJ_ERR_INVALID, "null argument");
    if (res->njoins > 1) fail(TJ_ERR_INVALID, "batched result: not supported");
    cudaStream_t st = (cudaStream_t)stream;
    TJ_CUDA(cudaMemsetAsync(counts_out, 0, (size_t)res->n_rows * 4, st));
    if (res->count > 0)
        neighbor_counts<<<(unsigned)((res->count + 255) / 256), 256, 0, st>>>(res->keys.p, res->count, res->n_cols,
                                                                               counts_out, flat_out);
    TJ_CUDA(cudaGetLastError());
    return TJ_OK;
    TJ_API_END
}

void tj_result_free(tj_result* res) {
    try {
        delete res;
    } catch (...) {
    }
}

int tj_index_build(const void* X, int64_t n, int32_t d, int32_t dtype, double eps2, tj_index** out, void* stream) {
    TJ_API_BEGIN
    if (!out || !X) fail(TJ_ERR_INVALID, "null argument");
    if (n <= 0 || d <= 0) fail(TJ_ERR_INVALID, "invalid shape");
    if (n >= (1ll << 32)) fail(TJ_ERR_INVALID, "more than 2^32 - 1 rows");
    if (dtype != TJ_DTYPE_F32 && dtype != TJ_DTYPE_I16) fail(TJ_ERR_INVALID, "unknown dtype");
    cudaStream_t st = (cudaStream_t)stream;
    stage_reset();
    std::unique_ptr<tj_index> ix(new tj_index());
    DBuf<Counters> ctr(1, st);
    launch(zero_counters, 1, 32, 0, st, ctr.p, 0);
    DBuf<FrameParams> fp(1, st);
    DBuf<float> center((size_t)d, st);
    const void* srcs[1] = {X};
    const long long ns[1] = {n};
    const bool pca_frame = compute_frame(srcs, ns, 1, d, dtype, kFrameAuto, fp.p, center.p, st);
    Side& s = ix->side;
    s.src = X; s.dtype = dtype; s.n = n; s.d = d; s.screen = kScreenPlain;
    prepare_side(s, fp.p, pca_frame, center.p, st, &ctr.p->status);
    tile_stats(s, kTileR, ix->t128, st);
    tile_stats(s, kTileS, ix->t256, st);
    const JoinParams jp = make_params(eps2, d, 64, 0, n, n, true);
    build_candidates(ix->t128, ix->t256, jp.Tp, true, 64, ix->cand, st);
    // cells: runs of equal Morton keys, prefix-sum offsets
    DBuf<uint32_t> flag((size_t)n, st), pos((size_t)n, st), ncell(1, st);
    DBuf<uint32_t> sws(scan_workspace_elems((size_t)n) + 4, st);
    launch(cell_flags, (unsigned)((n + 255) / 256), 256, 0, st, s.keys.p, n, flag.p);
    exclusive_scan_u32(flag.p, pos.p, (size_t)n, ncell.p, sws.p, st);
    uint32_t hc[3] = {0, 0, 0};
    TJ_CUDA(cudaMemcpyAsync(&hc[0], ncell.p, 4, cudaMemcpyDeviceToHost, st));
    TJ_CUDA(cudaMemcpyAsync(&hc[1], ix->cand.dev_counts.p, 8, cudaMemcpyDeviceToHost, st));
    Counters h;
    TJ_CUDA(cudaMemcpyAsync(&h, ctr.p, sizeof(Counters), cudaMemcpyDeviceToHost, st));
    TJ_CUDA(cudaStreamSynchronize(st));
    check_status(h.status);
    ix->n_cells = hc[0];
    ix->n_tile_pairs = hc[1];
    ix->cand.total = hc[1];
    ix->cand.nchunks = hc[2];
    ix->cell_start = DBuf<uint32_t>((size_t)ix->n_cells + 1, st);
    launch(cell_starts, (unsigned)((n + 255) / 256), 256, 0, st, flag.p, pos.p, n, ix->cell_start.p, ncell.p);
    TJ_CUDA(cudaGetLastError());
    TJ_CUDA(cudaStreamSynchronize(st));
    *out = ix.release();
    return TJ_OK;
    TJ_API_END
}

int tj_index_info(const tj_index* idx, int64_t* n_cells, int64_t* n_tiles, int64_t* n_candidate_tile_pairs) {
    if (!idx) { g_last_error = "null index"; return TJ_ERR_INVALID; }
    if (n_cells) *n_cells = idx->n_cells;
    if (n_tiles) *n_tiles = idx->t128.ntiles;
    if (n_candidate_tile_pairs) *n_candidate_tile_pairs = idx->n_tile_pairs;
    return TJ_OK;
}

int tj_index_copy(const tj_index* idx, uint32_t* perm, uint64_t* keys, uint32_t* cell_start, uint32_t* tile_pairs,
                  void* stream) {
    TJ_API_BEGIN
    if (!idx) fail(TJ_ERR_INVALID, "null index");
    cudaStream_t st = (cudaStream_t)stream;
    const size_t n = (size_t)idx->side.n;
    if (perm) TJ_CUDA(cudaMemcpyAsync(perm, idx->side.perm.p, n * 4, cudaMemcpyDeviceToDevice, st));
    if (keys) TJ_CUDA(cudaMemcpyAsync(keys, idx->side.keys.p, n * 8, cudaMemcpyDeviceToDevice, st));
    if (cell_start)
        TJ_CUDA(cudaMemcpyAsync(cell_start, idx->cell_start.p, ((size_t)idx->n_cells + 1) * 4,
                                cudaMemcpyDeviceToDevice, st));
    if (tile_pairs && idx->n_tile_pairs > 0) {
        launch(tile_pair_list, num_sms() * 4, 256, 0, st, idx->cand.chunks.p, idx->cand.dev_counts.p + 1,
                                                       idx->cand.jlist.p, tile_pairs);
        TJ_CUDA(cudaGetLastError());
    }
    return TJ_OK;
    TJ_API_END
}

void tj_index_free(tj_index* idx) {
    try {
        delete idx;
    } catch (...) {
    }
}

int tj_join_batched(const tj_batch_join* joins, int32_t njoins, int32_t screen, const tj_options* opt,
                    tj_result** out, void* stream) {
    TJ_API_BEGIN
    if (!out || (njoins > 0 && !joins)) fail(TJ_ERR_INVALID, "null argument");
    *out = nullptr;
    if (njoins < 1) fail(TJ_ERR_INVALID, "njoins must be >= 1");
    if (screen < 0 || screen > 5 || screen == TJ_SCREEN_INT8LIMB) fail(TJ_ERR_UNSUPPORTED, "batched joins take FP32 screens");
    check_flags(opt);
    std::vector<JoinIn> js((size_t)njoins);
    for (int k = 0; k < njoins; ++k) js[k] = JoinIn{joins[k].R, joins[k].S, joins[k].nR, joins[k].nS, joins[k].d, joins[k].eps2};
    std::unique_ptr<tj_result> res(new tj_result());
    run_batch(js, TJ_DTYPE_F32, TJ_MODE_RS, screen, opt, res.get(), (cudaStream_t)stream);
    if (res->offsets.empty()) res->offsets.assign((size_t)njoins + 1, res->count);   // one join: [0, count)
    if (njoins == 1) res->offsets[0] = 0;
    *out = res.release();
    return TJ_OK;
    TJ_API_END
}

int tj_batch_offsets(const tj_result* res, int64_t* offsets_host) {
    if (!res || !offsets_host) { g_last_error = "null argument"; return TJ_ERR_INVALID; }
    if (res->offsets.empty()) { g_last_error = "not a batched result"; return TJ_ERR_INVALID; }
    memcpy(offsets_host, res->offsets.data(), res->offsets.size() * sizeof(int64_t));
    return TJ_OK;
}

int tj_batch_pairs(const tj_result* res, int64_t* i_out, int64_t* j_out, void* stream) {
    TJ_API_BEGIN
    if (!res) fail(TJ_ERR_INVALID, "null result");
    if (res->count == 0) return TJ_OK;
    if (!i_out || !j_out) fail(TJ_ERR_INVALID, "null output");
    if (res->njoins == 1) {
        decode_pairs(res->keys.p, res->count, res->n_cols, i_out, j_out, (cudaStream_t)stream);
        return TJ_OK;
    }
    decode_pairs_batched(res->keys.p, res->count, res->d_keyoff.p, res->d_cols.p, res->njoins, i_out, j_out,
                         (cudaStream_t)stream);
    return TJ_OK;
    TJ_API_END
}

int tj_set_wait_limit(int64_t ns) {
    if (ns < 0) { g_last_error = "the wait limit must be >= 0"; return TJ_ERR_INVALID; }
    g_wait_ns = ns == 0 ? kWaitLimitNs : (unsigned long long)ns;
    return TJ_OK;
}

const char* tj_last_error_string(void) { return g_last_error.c_str(); }

int tj_version(void) { return 1; }

int64_t tj_kernel_launches(void) { return (int64_t)g_launches.load(); }

int tj_device_sm_count(void) {
    try {
        return num_sms();
    } catch (...) {
        return -1;
    }
}

int tj_pool_usage(int64_t* reserved, int64_t* used, int64_t* reserved_high) {
    TJ_API_BEGIN
    cudaMemPool_t pool = pool_for_current();
    uint64_t v = 0;
    if (reserved) {
        TJ_CUDA(cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReservedMemCurrent, &v));
        *reserved = (int64_t)(v + workspace_bytes());
    }
    if (used) { TJ_CUDA(cudaMemPoolGetAttribute(pool, cudaMemPoolAttrUsedMemCurrent, &v)); *used = (int64_t)v; }
    if (reserved_high) {
        TJ_CUDA(cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReservedMemHigh, &v));
        *reserved_high = (int64_t)v;
    }
    return TJ_OK;
    TJ_API_END
}

int tj_pool_reserve(int64_t bytes, void* stream) {
    TJ_API_BEGIN
    if (bytes < 0) fail(TJ_ERR_INVALID, "bytes must be >= 0");
    cudaMemPool_t pool = pool_for_current();
    uint64_t have = 0;
    TJ_CUDA(cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReservedMemCurrent, &have));
    if ((uint64_t)bytes > have) {
        cudaStream_t st = (cudaStream_t)stream;
        void* p = dalloc((size_t)bytes, st);
        dfree(p, st);
        TJ_CUDA(cudaStreamSynchronize(st));
    }
    return TJ_OK;
    TJ_API_END
}

int tj_pool_trim(int64_t keep_bytes) {
    TJ_API_BEGIN
    if (keep_bytes < 0) fail(TJ_ERR_INVALID, "keep_bytes must be >= 0");
    release_cached(nullptr);
    TJ_CUDA(cudaDeviceSynchronize());   // frees pending on any stream complete before the trim
    TJ_CUDA(cudaMemPoolTrimTo(pool_for_current(), (size_t)keep_bytes));
    return TJ_OK;
    TJ_API_END
}

}  // extern "C"
