// Internal host-side interface between the pipeline stages of libtensorjoin.
#pragma once

#include <cstddef>
#include <cstdint>
#include <cstring>
#include <string>
#include <utility>
#include <vector>

#include "tj_common.cuh"

namespace tj {

// ------------------------------------------------------------------ errors
struct Error {
    int code;
    std::string msg;
};
[[noreturn]] void fail(int code, const std::string& msg);
void set_last_error(const std::string& msg);
void check_cuda(cudaError_t e, const char* what);
#define TJ_CUDA(x) ::tj::check_cuda((x), #x)

// ------------------------------------------------------------------ device memory (tj_memory.cu)
// dalloc/dfree: while a WorkspaceScope is open on this thread and device, blocks come from the
// join workspace (a stack reclaimed in free order; overflow goes to the pool); otherwise from the
// stream-ordered pool.  Result buffers, which outlive the join, use result_alloc/result_release
// (a small cache of released result buffers in front of the pool).
cudaMemPool_t pool_for_current();
void* dalloc(size_t bytes, cudaStream_t st);
void dfree(void* p, cudaStream_t st);
void* result_alloc(size_t bytes, cudaStream_t st, size_t* cap_out);
void result_release(void* p, size_t cap, cudaStream_t st);
void release_cached(cudaStream_t st);   // drop cached result buffers and this thread's workspace
size_t workspace_bytes();               // this thread's workspace on the current device

// Opens the join workspace for the lifetime of the object (one join, all work on stream `st`).
// Closing it re-makes the workspace if the join needed more than it held.
struct WorkspaceScope {
    cudaStream_t st;
    int dev;
    explicit WorkspaceScope(cudaStream_t s);
    ~WorkspaceScope();
    WorkspaceScope(const WorkspaceScope&) = delete;
    WorkspaceScope& operator=(const WorkspaceScope&) = delete;
};
// Allocations made while this object lives bypass the workspace (buffers that leave the join).
struct WorkspaceSuspend {
    int dev;
    WorkspaceSuspend();
    ~WorkspaceSuspend();
    WorkspaceSuspend(const WorkspaceSuspend&) = delete;
    WorkspaceSuspend& operator=(const WorkspaceSuspend&) = delete;
};

template <class T>
struct DBuf {
    T* p = nullptr;
    size_t n = 0;
    cudaStream_t st = nullptr;
    size_t rcap = 0;   // > 0: a result buffer of rcap bytes (goes back to the result cache)
    DBuf() = default;
    DBuf(size_t n_, cudaStream_t s) : n(n_), st(s) { p = n ? (T*)dalloc(n * sizeof(T), s) : nullptr; }
    // a buffer that may leave the join as part of a result
    static DBuf result(size_t n_, cudaStream_t s) {
        DBuf b;
        b.n = n_;
        b.st = s;
        b.p = (T*)result_alloc(n_ * sizeof(T), s, &b.rcap);
        return b;
    }
    DBuf(const DBuf&) = delete;
    DBuf& operator=(const DBuf&) = delete;
    DBuf(DBuf&& o) noexcept : p(o.p), n(o.n), st(o.st), rcap(o.rcap) { o.p = nullptr; o.n = 0; o.rcap = 0; }
    DBuf& operator=(DBuf&& o) noexcept {
        if (this != &o) {
            reset();
            p = o.p; n = o.n; st = o.st; rcap = o.rcap;
            o.p = nullptr; o.n = 0; o.rcap = 0;
        }
        return *this;
    }
    ~DBuf() { reset(); }
    void reset() {
        if (p) {
            if (rcap) result_release(p, rcap, st);
            else dfree(p, st);
        }
        p = nullptr;
        n = 0;
        rcap = 0;
    }
    size_t bytes() const { return n * sizeof(T); }
};

// Host -> device copy of a small host table through a per-thread pinned staging arena, so the copy
// is asynchronous (a pageable source would make cudaMemcpyAsync wait for the stream).  Staging
// regions are reused only after stage_reset(), which waits for the last staged copy.
void upload(void* dev_dst, const void* host_src, size_t bytes, cudaStream_t st);
void stage_reset();

// ------------------------------------------------------------------ scan / sort (tj_sort.cu)
size_t scan_workspace_elems(size_t n);
void exclusive_scan_u32(const uint32_t* in, uint32_t* out, size_t n, uint32_t* total, uint32_t* ws,
                        cudaStream_t st);
size_t radix_workspace_elems(size_t n);
void radix_sort(uint64_t* keys, uint32_t* vals, uint64_t* keys_tmp, uint32_t* vals_tmp, size_t n, int bits,
                uint32_t* ws, cudaStream_t st, unsigned long long* status = nullptr, bool* in_tmp = nullptr);
int radix_passes(int bits);
// True when radix_sort with a status word and in_tmp leaves the sorted keys in the temporaries.
bool radix_result_in_tmp(size_t n, int bits);

// ------------------------------------------------------------------ enums (mirror include/tensorjoin.h)
enum DType { kF32 = 0, kI16 = 1 };
enum Mode { kModeRS = 0, kModeUpper = 1, kModeDirected = 2 };
enum Screen { kScreenPlain = 0, kScreenBF16 = 1, kScreenFP16 = 2, kScreenInt8Limb = 3, kScreenBF16X3 = 4, kScreenFP16X3 = 5 };

// ------------------------------------------------------------------ prepared side (tj_index.cu)
// A side of the join in Morton order: permutation, MMA operand and per-row certificate metadata.
// Row r of every array is the point perm[r] of the caller's input.
struct Side {
    const void* src = nullptr;   // caller's input rows, original order (not owned)
    int dtype = kF32;
    long long n = 0;             // rows
    int d = 0;
    int screen = kScreenBF16;
    int kpad = 0;                // operand row length in elements (multiple of 64; int8: 128)
    int split = 0;               // 1: operand rows are [z_hi | z_lo] (2 * kpad elements)
    long long rows_pad = 0;      // operand rows (multiple of 256)
    DBuf<uint32_t> perm;         // [n] sorted position -> row of the side's source matrix
    DBuf<uint32_t> perm_local;   // [n] sorted position -> row id inside its own join (batched sides)
    const uint32_t* emit = nullptr;   // ids written into pair keys: perm (one join) or perm_local
    const long long* d_rowoff = nullptr;   // device [njc + 1]: first source row of each join (batched)
    int njc = 1;                 // joins concatenated in this side
    DBuf<uint64_t> keys;         // [n] Morton keys (sorted)
    DBuf<uint16_t> op;           // [rows_pad, kpad or 2*kpad] bf16 / fp16 operand of x - centre
    DBuf<int8_t> op8;            // [rows_pad, 2*kpad] int8 limbs [hi | lo] (int8 limb screen)
    DBuf<float> xs;              // [rows_pad, d] FP32 rows in sorted order (plain screen)
    DBuf<double> nrm2;           // [rows_pad] sequential FP64 sum of squares of x
    DBuf<float> nrm2f;           // [rows_pad] FP32 nearest of nrm2
    DBuf<float> zn;              // [rows_pad] upper bound of ||z|| (z = operand row)
    DBuf<float> en;              // [rows_pad] upper bound of ||x - z||
    DBuf<float> yn;              // [rows_pad] upper bound of ||x - centre||
    DBuf<float> zl;              // [rows_pad] upper bound of ||z_lo|| (0 without the split)
    DBuf<long long> inorm;       // [rows_pad] exact integer squared norms (int path)
};

// Tile statistics at one tile granularity (128 rows for R, 256 rows for S).
struct TileSet {
    int tile = 0;
    int ntiles = 0;
    int d = 0;
    DBuf<float> ctrT;      // [d][ntiles] centroid (transposed for coalesced candidate tests)
    DBuf<float> loT, hiT;  // [d][ntiles] exact per-dimension min / max
    DBuf<float> rad;       // [ntiles] upper bound of max ||x - centroid||
    DBuf<float> maxZ, maxE, maxY, maxB, beta, maxZl;  // [ntiles] maxima of the row bounds
    DBuf<uint32_t> nvalid;  // [ntiles] rows of the tile that are real points
    DBuf<uint32_t> row0;    // [ntiles] first sorted row of the tile
    std::vector<uint32_t> h_row0, h_nvalid, h_join;   // host tile tables (batched sides; empty: uniform tiles)
    bool built = false;   // statistics already computed (by the fused operand pass)
    DBuf<float> ctrR, loR, hiR;   // [ntiles][d] row-major copies (half tiles: the half-mask test)
};

// Candidate tile pairs grouped by R tile, cut into chunks scheduled J-window-major.
struct Candidates {
    DBuf<uint32_t> cnt;       // [ntR] candidates per R tile
    DBuf<uint32_t> off;       // [ntR] exclusive prefix of cnt
    DBuf<uint32_t> jlist;     // [total] S tile ids, ascending within each R tile
    DBuf<uint4> chunks;       // [nchunks] (I, begin, end, 0) in execution order
    DBuf<uint32_t> dev_counts;  // [2]: total candidates, total chunks (device)
    uint32_t total = 0;       // host copies (filled after a sync)
    uint32_t nchunks = 0;
    size_t chunks_cap = 0;
};

constexpr int kPcaMaxD = 128;   // principal-component frames for 9 <= d <= kPcaMaxD
struct FrameParams {
    int m = 0;               // indexed dimensions (or principal directions)
    int bits = 0;            // bits per indexed dimension
    int pca = 0;             // 1: cells over the projections onto the top m principal directions
    int dims[16] = {0};      // pca == 0: the indexed input dimensions
    float lo[16] = {0};
    float inv_w[16] = {0};
    float V[8 * kPcaMaxD] = {0};   // pca == 1: direction k is V[k * d .. k * d + d)
};

// side preparation
// Index frame shared by both sides: cells over the m = min(d, 8) highest-variance input
// dimensions, or cells over the top 8 principal directions of a sampled covariance
// (kFramePca: whenever 9 <= d <= kPcaMaxD; kFrameAuto: also needs kPcaMinRows rows in all). The
// return value says whether the principal-component frame was built. Also writes the
// per-dimension centre.
constexpr int kFrameAuto = 0, kFrameAxes = 1, kFramePca = 2;
constexpr long long kPcaMinRows = 1ll << 17;   // below this the frame's fixed cost is not repaid
bool compute_frame(const void* const* srcs, const long long* ns, int nsrc, int d, int dtype, int frame_mode,
                   FrameParams* fp, float* center, cudaStream_t st);
// Morton sort and operand preparation of one side.  With a tile set (tile 128 or 256, host tables
// filled when the tiling is not uniform) the operands and that tiling's statistics come from one
// fused pass where the side allows it (16-bit screens, FP32 rows, d % 4 == 0, d <= 128), and
// `halves` (256-row tiles only) receives the statistics of their 128-row halves; the tile sets are
// then marked built and tile_stats leaves them alone.
void prepare_side(Side& s, const FrameParams* fp_dev, bool pca_frame, const float* center, cudaStream_t st,
                  unsigned long long* status, TileSet* ts = nullptr, int tile = 0, TileSet* halves = nullptr);
void tile_stats(const Side& s, int tile, TileSet& ts, cudaStream_t st);
void build_candidates(const TileSet& tr, const TileSet& ts, double T, bool self_join, int chunk_items,
                      Candidates& c, cudaStream_t st);
void gather_rows(const std::vector<const void*>& srcs, const std::vector<long long>& rows, int d, int esize,
                 void* dst, cudaStream_t st);
void compute_perm_local(Side& s, cudaStream_t st);

// Candidate tile pairs of many joins at once (block-diagonal: tiles only pair within their join).
struct CandBlock {              // one cand_test block: up to 16 R tiles of one join against all its S tiles
    uint32_t i0, ni;            // first global R tile, tiles in the block
    uint32_t j0, nj;            // first global S tile of the join, S tiles of the join
    uint32_t cls, pad;          // class of the join (selects the tile statistics arrays)
};
struct CandClassView {          // tile statistics of one class, indexed by class-local tile ids
    const float *rctrT, *rloT, *rhiT, *rrad, *sctrT, *sloT, *shiT, *srad;
    int ntR, ntS, rbase, sbase, d, pad;
};
void build_candidates_batched(const std::vector<CandClassView>& classes, const std::vector<CandBlock>& blocks,
                              const std::vector<double>& Tp_per_block, int ntR_total, int words, int chunk_items,
                              const std::vector<uint32_t>& rtile_sbase, Candidates& c, cudaStream_t st);

// Half-tile masks (one-SM tensor-core screen): R tile statistics and 128-row S half-tile statistics
// of one class, class-local indices; ntH = 2 x the class's 256-row S tiles.
struct HalfView {
    const float *rctrT, *rloT, *rhiT, *rrad;   // R tiles: [d][ntR]
    const float *hctrR, *hloR, *hhiR, *hrad;   // halves: [ntH][d] (row-major)
    const uint32_t* hnv;   // [ntH] rows of each half that are real points
    int ntR, ntH, rbase, sbase, d, pad;
};
// Marks the live 128-row halves of every candidate's S tile in bits 30-31 of its jlist entry.
void half_masks(const std::vector<HalfView>& views, const Candidates& c, int ntR_total, const uint4* rtiles,
                const JoinParams* jps, bool self_join, cudaStream_t st);
// Row-major copies (ctrR, loR, hiR) of a tile set's centroids and boxes.
void tile_stats_rowmajor(TileSet& ts, cudaStream_t st);
constexpr uint32_t kJMask = 0x3FFFFFFFu;   // jlist entry: S tile id in the low 30 bits

// ------------------------------------------------------------------ screen / refine / emit
struct EmitBuffers {
    uint64_t* acc = nullptr;   // accept keys
    unsigned long long acc_cap = 0;
    uint64_t* band = nullptr;  // band keys (canonical key of the pair)
    unsigned long long band_cap = 0;
    Counters* ctr = nullptr;
};

constexpr int kMaxClass = 4;

// Everything a screen launch needs: up to kMaxClass classes (same d inside a class) of prepared
// sides, global R / S tile tables (row0, nvalid, join, class), the global chunk list, per-join
// parameters, and per-join source pointers for the FP64 refinement.
struct ScreenInput {
    int ncls = 0;
    const Side* R[kMaxClass] = {};
    const Side* S[kMaxClass] = {};
    const TileSet* tR[kMaxClass] = {};
    const TileSet* tS[kMaxClass] = {};
    int rbase[kMaxClass] = {}, sbase[kMaxClass] = {};   // global tile id of each class's first tile
    int ntR_total = 0, ntS_total = 0;
    const uint4* rtiles = nullptr;      // device [ntR_total]: (row0 in class, nvalid, join, class)
    const uint4* stiles = nullptr;      // device [ntS_total]
    const Candidates* cand = nullptr;
    const JoinParams* jps = nullptr;    // device [njoins]
    const JoinParams* h_jps = nullptr;  // host copy of the same table
    int njoins = 0;
    const unsigned long long* key_off = nullptr;   // device [njoins]: ascending key offsets
    const void* const* rsrc = nullptr;  // device [njoins]: caller's R rows of each join
    const void* const* ssrc = nullptr;  // device [njoins]
    long long T_int = 0;                // integer threshold (int8-limb screen, single join)
    bool allow_pair = true;             // the CTA-pair tensor-core screen may be used where it applies
    bool i8_four_products = false;      // int8-limb screen: all four limb products (exact in the kernel)
    bool half_packed = false;           // jlist entries carry live-half masks (one-SM 16-bit screens)
    int k_block = 0;                    // 16-bit screens: elements per k-block (16 / 32 / 64; 0: by d)
    int stages = 0;                     // 16-bit screens: operand stages in flight (0: all compiled)
    mutable bool used_pair = false;     // set by screen_tc
    JoinParams jp0{};                   // host copy of join 0's parameters (single-join kernels)
    // screen-error diagnostics (tensor-core screens): sampled accumulators and the analysis result
    float* dump = nullptr;              // [dump_items][128][256]
    uint4* dump_ids = nullptr;          // [dump_items]
    unsigned dump_every = 0, dump_items = 0;
    unsigned long long* diag_out = nullptr;   // [3]: max |d2hat - d2| (double bits), max ratio to bound, pairs
    // TJ_FLAG_SCREEN_TIMES (tensor-core screens): per-join first-start / last-end and per-CTA start / end
    // %globaltimer stamps, null when off
    unsigned long long* join_t = nullptr;     // [2 njoins]
    unsigned long long* cta_t = nullptr;      // [2 * grid]
    unsigned long long* role_t = nullptr;     // [16] stall accounting of the 16-bit screens (SM cycles)
};

void screen_tc(const ScreenInput& g, const EmitBuffers& eb, cudaStream_t st);
void screen_plain(const ScreenInput& g, const EmitBuffers& eb, cudaStream_t st);
void screen_i8(const ScreenInput& g, const EmitBuffers& eb, cudaStream_t st);
// true when screen_i8 runs the high-limb screen (hh products only; undecided pairs go to the band
// and the exact integer refinement), false for the four-product screen (exact, no band)
bool i8_high_limb_screen(const ScreenInput& g);
// FP64 terminal for the band; fp32_stage puts the certified FP32 band stage in front of it.
void refine_band(const ScreenInput& g, const EmitBuffers& eb, bool fp32_stage, cudaStream_t st);
void expand_directed(const uint64_t* upper, unsigned long long n_upper_slots, uint64_t* out, long long N,
                     cudaStream_t st);
void decode_pairs(const uint64_t* keys, long long n, long long n_cols, int64_t* i_out, int64_t* j_out,
                  cudaStream_t st);
void decode_pairs_batched(const uint64_t* keys, long long n, const unsigned long long* key_off,
                          const long long* n_cols, int njoins, int64_t* i_out, int64_t* j_out, cudaStream_t st);
void batch_offsets(const uint64_t* keys, long long n, const unsigned long long* key_off, int njoins,
                   long long* offsets, cudaStream_t st);

int num_sms();
// limit of the screen kernels' pipeline waits for joins started on the calling thread (tj_set_wait_limit)
unsigned long long pipeline_wait_ns();

// Every kernel of the library is launched through launch(): it checks the launch and counts it
// (tj_kernel_launches() reports the running total, used to audit what ran inside a timed region).
void count_launch();
template <class... KArgs, class... Args>
void launch(void (*k)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t st, Args&&... args) {
    k<<<grid, block, smem, st>>>(std::forward<Args>(args)...);
    count_launch();
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {   // name the kernel's resources in the error
        cudaFuncAttributes fa;
        memset(&fa, 0, sizeof(fa));
        cudaFuncGetAttributes(&fa, k);
        cudaGetLastError();
        fail(-2, std::string("kernel launch: ") + cudaGetErrorString(e) + " (block " +
                     std::to_string(block.x * block.y * block.z) + " threads, " + std::to_string(smem) +
                     " B dynamic shared; kernel: " + std::to_string(fa.numRegs) + " registers, max " +
                     std::to_string(fa.maxThreadsPerBlock) + " threads, " + std::to_string(fa.sharedSizeBytes) +
                     " B static shared, " + std::to_string(fa.maxDynamicSharedSizeBytes) + " B dynamic allowed)");
    }
}

}  // namespace tj
