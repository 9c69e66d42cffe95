/*
 * libtensorjoin -- B200 (sm_100a) certified exact epsilon-join, C ABI.
 *
 * Every function returns 0 (TJ_OK) or a negative TJ_ERR_* code; the message of
 * the last failure on the calling thread is available from
 * tj_last_error_string().  No C++ exception crosses this boundary.  Device
 * pointers are plain CUDA device addresses (e.g. from torch tensors), `stream`
 * is a cudaStream_t passed as void*, and the library never frees caller memory.
 * Handles (tj_result, tj_index) own their device memory until freed; calls on
 * distinct handles are independent (no global result state).
 *
 * Predicate (every mode): a pair (i, j) is in the result iff
 *     sum_{k=0..d-1} (double(R[i,k]) - double(S[j,k]))^2  <= eps2
 * evaluated in FP64 in sequential k order (int16 inputs: exact integers).
 * Results are sorted ascending by (i, j); canonical key = i * n_cols + j.
 *
 * Reference interfaces replaced (wangwenqingqq/tensorjoin-variants, paths inside
 * tensorjoin_20260902_certified_exact_join/):
 *   - the script-level join contract: FP32 rows in, sorted uint64 canonical ids
 *     out (src/g2b_public_common.py:97-143, src/run_g2b_tensorjoin_public.py:139-395;
 *     R-S driver src/run_d1_triton.py:290-420);
 *   - GDS-Join's ctypes library API GDSJoinPy / copyResultIntoPythonArray
 *     (adapters/gds_g2a/main.cu:360, :488-510; adapters/gds_g2a/gdsjoingpu.py:146-232);
 *   - the output-stage library output_mirror / output_sort
 *     (tensorjoin_20260908_output_audit/src/output.cu:19-31).
 */
#ifndef TENSORJOIN_H
#define TENSORJOIN_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define TJ_OK 0
#define TJ_ERR_INVALID (-1)     /* bad argument (null pointer, d <= 0, unknown mode, ...) */
#define TJ_ERR_CUDA (-2)        /* a CUDA runtime/driver call failed */
#define TJ_ERR_INPUT (-3)       /* NaN / Inf or a row norm beyond 2^50 in the input */
#define TJ_ERR_RANGE (-4)       /* input magnitude outside the FP16 operand range (use BF16) */
#define TJ_ERR_TIMEOUT (-5)     /* a bounded device wait expired (kernel returned early) */
#define TJ_ERR_NOMEM (-6)       /* device allocation failed */
#define TJ_ERR_UNSUPPORTED (-7) /* combination not supported (e.g. int16 with a float screen) */

/* input element type */
#define TJ_DTYPE_F32 0
#define TJ_DTYPE_I16 1          /* int14 values in [-8192, 8191] stored as int16 */

/* join mode */
#define TJ_MODE_RS 0            /* all (i, j), i in R, j in S */
#define TJ_MODE_UPPER 1         /* self-join (S == R), pairs i < j */
#define TJ_MODE_DIRECTED 2      /* self-join, all (i, j) incl. the n self pairs (reference canonical form) */

/* distance screen */
#define TJ_SCREEN_PLAIN 0       /* FP32 direct difference (no tensor cores) + FP64 refinement of the band */
#define TJ_SCREEN_BF16 1        /* tcgen05 BF16 x BF16 -> FP32 screen + certified band + FP64 refinement */
#define TJ_SCREEN_FP16 2        /* tcgen05 FP16 x FP16 -> FP32 screen + certified band + FP64 refinement */
#define TJ_SCREEN_INT8LIMB 3    /* int14 via two int8 limbs, exact INT32 tensor-core products (int16 input) */
#define TJ_SCREEN_BF16X3 4      /* BF16 hi + lo operand limbs, 3 products per k into one FP32 accumulator */
#define TJ_SCREEN_FP16X3 5      /* FP16 hi + lo operand limbs, 3 products per k into one FP32 accumulator */

typedef struct tj_result tj_result;
typedef struct tj_index tj_index;

typedef struct tj_options {
    int64_t initial_capacity;   /* accept / band buffer slots for the first attempt (0: library default) */
    int32_t chunk_items;        /* tile pairs per scheduling chunk (0: 64) */
    int32_t flags;              /* TJ_FLAG_* bits */
    /* Tile-shape knobs of the 16-bit tensor-core screens (0: the library's choice; the pairs never
     * change): k_block = elements of K per pipeline stage (64, 32 or 16; must divide the padded row
     * length, which is a multiple of 64 for d > 32), stages = operand stages in flight (2 up to the
     * compiled 4, or 6 on the CTA pair; the hi/lo split compiles 2). */
    int32_t k_block;
    int32_t stages;
} tj_options;

/* Sample tile pairs during the tensor-core screen and report the screen's distance error against
 * sequential FP64 distances (tj_stats.screen_*).  Diagnostic: adds a sampling pass. */
#define TJ_FLAG_SCREEN_DIAG 1
/* Use the one-SM tensor-core screen even where the CTA-pair screen (cta_group::2, 256 x 256 tiles
 * over two SMs; one join, rows of >= 256 elements, every tile pair a candidate) would run. */
#define TJ_FLAG_SCREEN_1SM 2
/* Index frame: the cells rows are sorted by before they are cut into tiles.  By default a single
 * join with 9 <= d <= 128 and at least 2^17 rows in all uses cells over the top 8 principal
 * directions of a sampled covariance; every other join uses cells over the 8 highest-variance
 * input dimensions.  FRAME_AXES forces the input-dimension cells, FRAME_PCA the principal-direction
 * cells wherever 9 <= d <= 128 (any size, packed joins included).  The frame only changes which
 * rows share a tile, never the pairs.  Setting both is an error. */
#define TJ_FLAG_FRAME_AXES 4
#define TJ_FLAG_FRAME_PCA 8
/* Certified FP32 band stage: every band pair is first decided, where it can be, by an FP32 sum of
 * squared FP32 differences against thresholds that bound its rounding error; only the pairs it
 * cannot decide go on to the sequential FP64 terminal (tj_stats.band_fp64 counts them).  The
 * pairs are the same either way.  No effect on the plain and int8-limb screens. */
#define TJ_FLAG_BAND_FP32 16
/* int8-limb screen: issue all four limb products (hh, hl + lh, ll) on the tensor cores and decide
 * every pair exactly inside the screen (no band).  By default, for rows of up to 256 elements, the
 * screen issues only the high-limb product hh, bounds the low-limb terms by Cauchy-Schwarz, decides
 * each candidate by an exact INT64 interval test, and sends the few undecided pairs to the exact
 * integer refinement (tj_stats.band).  The pairs are the same either way. */
#define TJ_FLAG_I8_FOUR_PRODUCTS 32
/* Guard regions: 512 words of a fixed pattern (every byte -17, the reference's fill for retained
 * buffers) right after the part of the accept, band, result-key and sort buffers that a stage may
 * write, checked after the stage; an overwritten guard fails the join with TJ_ERR_CUDA.  A bounds
 * check in place of a memory sanitizer; costs four tiny launches per stage. */
#define TJ_FLAG_GUARDS 64
/* Keep the screen's own decisions in the result: its certified accepts and its band, before the
 * refinement, each sorted (tj_result_stage_keys).  For auditing each stage against an oracle. */
#define TJ_FLAG_STAGE_KEYS 128
/* Tensor-core screens: record %globaltimer stamps of every join's first chunk start and last chunk
 * end and of every CTA's start and end, and report their spread (tj_stats.join_span_ms_*,
 * screen_cta_tail_ms).  Diagnostic: one atomic per chunk and epilogue warp. */
#define TJ_FLAG_SCREEN_TIMES 256
/* One-SM 16-bit screens: issue both 128-row halves of every candidate tile pair.  By default each
 * half of a candidate's 256-row S tile is first tested against the R tile (the candidate test's
 * bounds on the half's own statistics) and only live halves are issued, packed densely into the
 * screen's MMA and epilogue pipeline.  The pairs are the same either way. */
#define TJ_FLAG_WHOLE_TILES 512

typedef struct tj_stats {
    int64_t n_rows, n_cols;       /* |R|, |S| (self-join: N, N) */
    int64_t pairs_all;            /* |R||S| (R-S) or N(N-1)/2 (self-join) */
    int64_t tile_pairs;           /* candidate tile pairs screened (128 x 256 each; one-SM 16-bit screens:
                                     those with a live 128-row half) */
    int64_t pairs_screened;       /* distance evaluations: sum over tile pairs of valid rows x valid cols */
    int64_t screen_accept;        /* pairs accepted by the certified screen alone */
    int64_t band;                 /* pairs sent to FP64 refinement */
    int64_t refine_accept;        /* band pairs accepted by FP64 refinement */
    int64_t rare_checks;          /* pairs that passed the screen's fast test without a certified accept
                                     (16-bit screens: the band the screen emits; int8-limb screens: the
                                     candidates that took the exact INT64 test) */
    int64_t result_pairs;         /* pairs in the output */
    int64_t retries;              /* capacity retries (overflow-and-retry passes) */
    double ms_index, ms_candidates, ms_screen, ms_refine, ms_sort, ms_total;   /* device time per stage */
    double screen_ops;            /* algorithmic screen operations: per pair 2d (16-bit), 6d (hi/lo split), 8d (int8 limbs) */
    double screen_max_abs_err;    /* TJ_FLAG_SCREEN_DIAG: max |(|x|^2 + |y|^2 - 2p) - d2_fp64| over the sampled pairs */
    double screen_err_over_bound; /* TJ_FLAG_SCREEN_DIAG: max of that error divided by the certified radius */
    int64_t screen_err_pairs;     /* TJ_FLAG_SCREEN_DIAG: sampled pairs */
    int64_t screen_pair;          /* 1 if the CTA-pair tensor-core screen ran */
    int64_t index_frame;          /* 1 if the index cells were over principal directions, 0 if over
                                     input dimensions */
    int64_t band_fp64;            /* band pairs decided by the FP64 terminal */
    double screen_ops_issued;     /* tensor-core operations the screen issued: 2 M N K per MMA over every
                                     tile pair it ran (padded rows, columns and K included) */
    /* TJ_FLAG_SCREEN_TIMES: spread of the CTAs' end times (the idle tail of the persistent screen), and
     * the median, 99th percentile and largest time from a join's first chunk start to its last chunk
     * end inside the screen launch */
    double screen_cta_tail_ms;
    double join_span_ms_p50, join_span_ms_p99, join_span_ms_max;
    /* TJ_FLAG_SCREEN_TIMES, one-SM and CTA-pair 16-bit screens: where each role of the persistent screen
     * spent its time, as fractions of that role's running time (SM clock cycles summed over the CTAs;
     * the epilogue's over its warps).  Producer: waiting for a free operand stage, for a free metadata
     * slot.  UMMA issuer: waiting for operands, for a free accumulator.  Epilogue: waiting for an
     * item's metadata, for its accumulator; reading and testing the accumulator; emitting (from the
     * warp scan to the last key written), and within that the output reservations. */
    double screen_prod_stage_wait, screen_prod_meta_wait;
    double screen_mma_operand_wait, screen_mma_acc_wait;
    double screen_epi_meta_wait, screen_epi_acc_wait, screen_epi_test, screen_epi_emit, screen_epi_reserve;
} tj_stats;

/* ----------------------------------------------------------------- joins */

/* Join R [nR, d] with S [nS, d] (device pointers, row-major, dtype elements).
 * mode TJ_MODE_RS uses S; the self-join modes ignore S (pass NULL or R).
 * eps2 is the threshold on the squared distance (eps * eps in FP64; an integer for int16 input).
 * On success *out receives a result handle (free with tj_result_free). */
int tj_join(const void* R, int64_t nR, const void* S, int64_t nS, int32_t d, int32_t dtype, double eps2,
            int32_t mode, int32_t screen, const tj_options* opt, tj_result** out, void* stream);

int64_t tj_result_count(const tj_result* res);
int tj_result_stats(const tj_result* res, tj_stats* out);
/* Sorted pairs as two int64 device arrays of tj_result_count() elements each. */
int tj_result_pairs(const tj_result* res, int64_t* i_out, int64_t* j_out, void* stream);
/* Sorted canonical keys i * n_cols + j (uint64 device array of tj_result_count() elements). */
int tj_result_keys(const tj_result* res, uint64_t* keys_out, void* stream);
/* TJ_FLAG_STAGE_KEYS results: stage 0 = the pairs the screen accepted by its certificate alone,
 * stage 1 = the band it passed to the refinement, as sorted canonical keys (self-joins: i < j, the
 * screen's form, also in directed mode).  *count receives the number of keys; keys_out (device,
 * *count elements) may be NULL to query the count.  No counterpart in the reference as an API; it
 * serves the per-stage audit the reference ran against its oracle
 * (src/run_g2a_tensorjoin.py:384-469). */
int tj_result_stage_keys(const tj_result* res, int32_t stage, uint64_t* keys_out, int64_t* count, void* stream);
/* GDS-style neighbour table: counts[n_rows] (uint32, device) and the flat j list (int64, device). */
int tj_result_neighbor_table(const tj_result* res, uint32_t* counts_out, int64_t* flat_out, void* stream);
void tj_result_free(tj_result* res);

/* ----------------------------------------------------------------- index */

/* Build the Morton-grid index of X [n, d] (device pointer): point permutation, cells with
 * prefix-sum offsets, and the 128-row tile statistics used for candidate pruning at threshold eps2. */
int tj_index_build(const void* X, int64_t n, int32_t d, int32_t dtype, double eps2, tj_index** out, void* stream);
int tj_index_info(const tj_index* idx, int64_t* n_cells, int64_t* n_tiles, int64_t* n_candidate_tile_pairs);
/* perm[n] (uint32: sorted position -> input row), keys[n] (uint64 Morton keys, sorted),
 * cell_start[n_cells + 1] (uint32 prefix offsets), candidate tile pairs as (I, J) uint32 pairs.
 * Any output pointer may be NULL. Device pointers. */
int tj_index_copy(const tj_index* idx, uint32_t* perm, uint64_t* keys, uint32_t* cell_start, uint32_t* tile_pairs,
                  void* stream);
void tj_index_free(tj_index* idx);

/* ----------------------------------------------------------------- batched ragged joins */

typedef struct tj_batch_join {
    const void* R;   /* device pointer [nR, d] */
    const void* S;   /* device pointer [nS, d] */
    int64_t nR, nS;
    int32_t d;
    int32_t pad;
    double eps2;
} tj_batch_join;

/* Run `njoins` independent R-S joins (FP32) in one persistent launch per stage.  The result holds
 * all joins' pairs; tj_batch_offsets gives each join's [start, end) range in the sorted output. */
int tj_join_batched(const tj_batch_join* joins, int32_t njoins, int32_t screen, const tj_options* opt,
                    tj_result** out, void* stream);
int tj_batch_offsets(const tj_result* res, int64_t* offsets_host /* njoins + 1 */);
int tj_batch_pairs(const tj_result* res, int64_t* i_out, int64_t* j_out, void* stream);

/* ----------------------------------------------------------------- allocation-free sort */

/* Sort n uint64 keys ascending by their low key_bits bits (1..64) into keys_out (device arrays;
 * keys_out may equal keys_in, or must not overlap it at all: a partial overlap returns
 * TJ_ERR_INVALID) without allocating any device memory.  No counterpart in the
 * reference: it is the canonical-order radix sort of this library, offered for callers that
 * cannot allocate at the call site (a fixed arena owned by the host engine, HBM reserved by
 * another allocator, or no allocation latency allowed between launches).  Its scratch is a
 * file-scope device array of about 9 MiB held by every GPU that loads the library; n is limited
 * to 1,048,576 keys (larger n returns TJ_ERR_INVALID).  All calls on a device share that array:
 * calls that overlap on the GPU race and must be serialised by the caller.  The first non-empty call
 * in a CUDA context resolves the array's address in that context (cudaGetSymbolAddress, cached per
 * context); make it before any stream capture.  n == 0 returns at once. */
int tj_sort_keys_noalloc(const uint64_t* keys_in, uint64_t* keys_out, int64_t n, int32_t key_bits, void* stream);

/* ----------------------------------------------------------------- misc */
/* Every wait inside the screen kernels is bounded: a kernel whose wait runs out sets a status bit,
 * lets its copies and tensor-core operations in flight finish (each of those waits bounded by 1 s),
 * frees its tensor memory and returns, and the join fails with TJ_ERR_TIMEOUT; the context stays
 * usable.  This sets the limit of the pipeline waits (between the copy, MMA and epilogue roles) for
 * joins started on the calling thread, in nanoseconds; 0 restores the default of 4 s.  No
 * counterpart in the reference (its kernels have no bounded waits).  Meant for tests of the timeout
 * path: a limit below the pipeline's normal latency makes joins fail. */
int tj_set_wait_limit(int64_t ns);
const char* tj_last_error_string(void);
int tj_version(void);
int tj_device_sm_count(void);
/* Running total of kernels this library has launched in the process (audit of timed regions). */
int64_t tj_kernel_launches(void);

/* Device memory held by the library on the current device.  No counterpart in the reference,
 * whose scripts allocated through torch.  A join takes its temporaries from a workspace owned by the
 * calling host thread (one block per thread and device, grown to 1.25x the largest join seen), its
 * result arrays from a cache of up to four buffers released by freed results, and everything else
 * from a stream-ordered pool; a steady stream of similar joins therefore maps no new memory.
 * tj_pool_usage: bytes held (pool reservation + this thread's workspace), bytes of the pool in live
 * allocations (results alive or cached), and the pool's peak reservation (any pointer may be NULL).
 * tj_pool_reserve: makes the pool hold at least `bytes` (one allocation and free on `stream`, then a
 * synchronisation of `stream`).
 * tj_pool_trim: frees the cached result buffers and this thread's workspace, waits for the device,
 * and returns pool memory above `keep_bytes` to the driver. */
int tj_pool_usage(int64_t* reserved, int64_t* used, int64_t* reserved_high);
int tj_pool_reserve(int64_t bytes, void* stream);
int tj_pool_trim(int64_t keep_bytes);

#ifdef __cplusplus
}
#endif

#endif /* TENSORJOIN_H */
