/*
 * CPU oracle for the certified exact epsilon-join.  TEST INFRASTRUCTURE ONLY:
 * it is imported by tests/, by __graft_entry__.smoke() and by bench.py's CPU
 * baseline leg as the checker; the product path never links or calls it.
 *
 * The predicate is the reference's exact CPU path restated as a fixed-order
 * loop:
 *
 *     d2(i, j) = sum_{k = 0 .. d-1} (double(x_ik) - double(y_jk))^2   (in k order)
 *     pair (i, j) is in the result  <=>  d2(i, j) <= T   (T = eps^2 in FP64)
 *
 * Reference semantics followed:
 *   - direct difference in FP64 of FP32 inputs widened to FP64:
 *     tensorjoin_20260902_certified_exact_join/src/run_g2a_tensorjoin.py:211-222
 *     (refine_ambiguous_fp64_i64) and adapters/gds_g2a/main.cu:962-965
 *     (CPUBruteForceTable's running sum);
 *   - T held in FP64, inclusive comparison `<= T`:
 *     src/prepare_g2_cifar.py:106-107, src/run_d1_triton.py:229;
 *   - canonical id encoding key = i * n_cols + j, sorted ascending
 *     (src/g2b_public_common.py:106-143, data/g2a_cifar4096/metadata.json);
 *   - self-join "directed" output includes the N self pairs and both (i, j)
 *     and (j, i) (src/prepare_g2_cifar.py:135-141); "upper" output is i < j.
 *
 * The summation order is sequential in k, one IEEE-754 double rounding per
 * subtract, multiply and add, with FMA contraction disabled
 * (-ffp-contract=off).  The GPU refinement kernel reproduces exactly this
 * order, so results are bit-identical.  Vectorisation is across pairs (eight
 * S rows at a time), never across k, so it does not change any pair's value.
 *
 * Integer inputs (int16 codes, the int14 configuration) use exact int64
 * arithmetic: d2 = sum (x - y)^2 <= T with T an integer.
 */
#include <math.h>
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#if defined(__FP_FAST_FMA) && !defined(ORACLE_ALLOW_FMA)
/* -ffp-contract=off is what matters; this guard only documents intent. */
#endif

typedef struct {
    uint64_t *keys;
    int64_t n;
    int64_t cap;
    int failed;
} keybuf;

static int kb_push(keybuf *b, uint64_t k) {
    if (b->n == b->cap) {
        int64_t nc = b->cap ? b->cap * 2 : 4096;
        uint64_t *p = (uint64_t *)realloc(b->keys, (size_t)nc * sizeof(uint64_t));
        if (!p) { b->failed = 1; return -1; }
        b->keys = p;
        b->cap = nc;
    }
    b->keys[b->n++] = k;
    return 0;
}

/* Sequential-k FP64 squared distance between two FP32 rows. */
static inline double seq_d2_f32(const float *x, const float *y, int d) {
    double acc = 0.0;
    for (int k = 0; k < d; ++k) {
        double t = (double)x[k] - (double)y[k];
        double sq = t * t;
        acc = acc + sq;
    }
    return acc;
}

/* Exact integer squared distance of two int16 rows in int64 (any int16 values: |x - y| <= 65535,
 * so each difference fits int32 and its square int64).  Integer addition is associative, so the
 * order of the sum does not matter and the compiler may vectorise it across k. */
static inline int64_t exact_d2_i16(const int16_t *x, const int16_t *y, int d) {
    int64_t acc = 0;
    for (int k = 0; k < d; ++k) {
        const int32_t t = (int32_t)x[k] - (int32_t)y[k];
        acc += (int64_t)t * (int64_t)t;
    }
    return acc;
}

/* mode: 0 = R-S (all i, j); 1 = self-join upper (i < j); 2 = self-join directed (all i, j incl. i == j) */
typedef struct {
    const void *R;
    const void *S;
    int64_t nR, nS;
    int d;
    double T;
    int64_t Ti;
    int mode;
    int is_int;
    int64_t row0, row1;
    keybuf out;
} job_t;

#define JB 8   /* S rows per block (transposed to k-major doubles) */
#define RB 16  /* R rows per block: each S block is loaded once per R block */

/* Four independent FP64 lanes (GCC vector extension): lane-wise IEEE operations, each lane one
 * pair's own accumulator, so the vectorisation is across pairs and never reorders a sum. */
typedef double v4d __attribute__((vector_size(32)));

static int cmp_u64(const void *a, const void *b) {
    const uint64_t x = *(const uint64_t *)a, y = *(const uint64_t *)b;
    return x < y ? -1 : x > y;
}

/* acc[r][jj] = sequential-k sum of (x_r[k] - blk[k][jj])^2 for two R rows and the JB S rows of blk. */
static inline void block_sums(const double *x0, const double *x1, const double *blk, int d, double out[2][JB]) {
    v4d a00 = {0, 0, 0, 0}, a01 = a00, a10 = a00, a11 = a00;
    for (int k = 0; k < d; ++k) {
        v4d b0, b1;
        memcpy(&b0, blk + (size_t)k * JB, sizeof(v4d));
        memcpy(&b1, blk + (size_t)k * JB + 4, sizeof(v4d));
        const v4d u = {x0[k], x0[k], x0[k], x0[k]};
        const v4d w = {x1[k], x1[k], x1[k], x1[k]};
        v4d t;
        t = u - b0; t = t * t; a00 = a00 + t;
        t = u - b1; t = t * t; a01 = a01 + t;
        t = w - b0; t = t * t; a10 = a10 + t;
        t = w - b1; t = t * t; a11 = a11 + t;
    }
    memcpy(out[0], &a00, sizeof(v4d));
    memcpy(out[0] + 4, &a01, sizeof(v4d));
    memcpy(out[1], &a10, sizeof(v4d));
    memcpy(out[1] + 4, &a11, sizeof(v4d));
}

/*
 * Rows [row0, row1) of R against S.  Blocks of RB R rows sweep S in blocks of JB rows, so S is
 * streamed from memory once per R block instead of once per R row; every pair still has its own
 * accumulator and its own sequential k order (the blocking changes which pairs are computed
 * together, never how one pair's sum is formed).  Keys of an R block are sorted before the next
 * block starts, so each thread's output stays ascending.
 *
 * int16 rows run through the same FP64 lanes: every difference (|t| <= 65535), square (< 2^32) and
 * partial sum (< d 2^32 <= 2^53 for d <= 2^21) is an integer that FP64 holds exactly, so the sum is
 * the exact integer squared distance, compared with the integer threshold after conversion.
 */
static void *worker(void *arg) {
    job_t *jb = (job_t *)arg;
    const int d = jb->d;
    const int64_t nS = jb->nS;
    double *blk = (double *)malloc((size_t)d * JB * sizeof(double));
    double *xr = (double *)malloc((size_t)d * (RB + 1) * sizeof(double));
    if (!blk || !xr) {
        free(blk); free(xr);
        jb->out.failed = 1;
        return NULL;
    }
    for (int64_t i0 = jb->row0; i0 < jb->row1; i0 += RB) {
        const int nr = (int)((jb->row1 - i0) < RB ? (jb->row1 - i0) : RB);
        const int64_t mark = jb->out.n;
        for (int r = 0; r < nr; ++r)
            for (int k = 0; k < d; ++k)
                xr[(size_t)r * d + k] = jb->is_int ? (double)((const int16_t *)jb->R)[(size_t)(i0 + r) * d + k]
                                                   : (double)((const float *)jb->R)[(size_t)(i0 + r) * d + k];
        for (int k = 0; k < d; ++k) xr[(size_t)nr * d + k] = 0.0;   /* partner of an odd last row */
        const int64_t jstart = (jb->mode == 1) ? i0 + 1 : 0;
        for (int64_t jb0 = jstart; jb0 < nS; jb0 += JB) {
            const int nb = (int)((nS - jb0) < JB ? (nS - jb0) : JB);
            for (int jj = 0; jj < JB; ++jj) {
                const size_t row = (size_t)(jb0 + (jj < nb ? jj : 0)) * d;
                for (int k = 0; k < d; ++k)
                    blk[(size_t)k * JB + jj] = jb->is_int ? (double)((const int16_t *)jb->S)[row + k]
                                                          : (double)((const float *)jb->S)[row + k];
            }
            for (int r = 0; r < nr; r += 2) {
                double acc[2][JB];
                block_sums(xr + (size_t)r * d, xr + (size_t)(r + 1) * d, blk, d, acc);
                for (int h = 0; h < 2 && r + h < nr; ++h) {
                    const int64_t i = i0 + r + h;
                    for (int jj = 0; jj < nb; ++jj) {
                        const int64_t j = jb0 + jj;
                        if (jb->mode == 1 && j <= i) continue;
                        const int in = jb->is_int ? ((int64_t)acc[h][jj] <= jb->Ti) : (acc[h][jj] <= jb->T);
                        if (in) kb_push(&jb->out, (uint64_t)i * (uint64_t)nS + (uint64_t)j);
                    }
                }
            }
        }
        if (jb->out.n - mark > 1)
            qsort(jb->out.keys + mark, (size_t)(jb->out.n - mark), sizeof(uint64_t), cmp_u64);
    }
    free(blk); free(xr);
    return NULL;
}

/* Row blocks balanced by pair count (the upper triangle makes early rows heavier). */
static void split_rows(int64_t nR, int64_t nS, int mode, int nt, int64_t *bounds) {
    bounds[0] = 0;
    if (mode != 1) {
        for (int t = 1; t <= nt; ++t) bounds[t] = nR * t / nt;
        return;
    }
    double total = (double)nR * (double)(nR - 1) / 2.0;
    int64_t r = 0;
    double acc = 0.0;
    for (int t = 1; t < nt; ++t) {
        double goal = total * t / nt;
        while (r < nR && acc < goal) { acc += (double)(nS - r - 1); ++r; }
        bounds[t] = r;
    }
    bounds[nt] = nR;
}

static int run(job_t *proto, int nthreads, uint64_t **out_keys, int64_t *out_count) {
    if (nthreads < 1) nthreads = 1;
    if (nthreads > 256) nthreads = 256;
    if (proto->nR < (int64_t)nthreads) nthreads = proto->nR > 0 ? (int)proto->nR : 1;
    job_t *jobs = (job_t *)calloc((size_t)nthreads, sizeof(job_t));
    pthread_t *th = (pthread_t *)calloc((size_t)nthreads, sizeof(pthread_t));
    int64_t *bounds = (int64_t *)calloc((size_t)nthreads + 1, sizeof(int64_t));
    if (!jobs || !th || !bounds) { free(jobs); free(th); free(bounds); return -1; }
    split_rows(proto->nR, proto->nS, proto->mode, nthreads, bounds);
    for (int t = 0; t < nthreads; ++t) {
        jobs[t] = *proto;
        jobs[t].row0 = bounds[t];
        jobs[t].row1 = bounds[t + 1];
        memset(&jobs[t].out, 0, sizeof(keybuf));
    }
    for (int t = 1; t < nthreads; ++t) pthread_create(&th[t], NULL, worker, &jobs[t]);
    worker(&jobs[0]);
    for (int t = 1; t < nthreads; ++t) pthread_join(th[t], NULL);
    int64_t total = 0;
    int failed = 0;
    for (int t = 0; t < nthreads; ++t) { total += jobs[t].out.n; failed |= jobs[t].out.failed; }
    uint64_t *keys = NULL;
    if (!failed) {
        keys = (uint64_t *)malloc((size_t)(total > 0 ? total : 1) * sizeof(uint64_t));
        if (!keys) failed = 1;
    }
    int64_t pos = 0;
    for (int t = 0; t < nthreads; ++t) {
        if (!failed && jobs[t].out.n) memcpy(keys + pos, jobs[t].out.keys, (size_t)jobs[t].out.n * sizeof(uint64_t));
        pos += jobs[t].out.n;
        free(jobs[t].out.keys);
    }
    free(jobs); free(th); free(bounds);
    if (failed) { free(keys); return -1; }
    *out_keys = keys;
    *out_count = total;
    return 0;
}

/*
 * Join two FP32 row-major matrices.  mode 0 = R-S, 1 = self upper (i < j),
 * 2 = self directed (includes i == j).  For modes 1 and 2, S must equal R.
 * Returns 0 and a malloc'd, ascending array of keys i * nS + j.
 */
int oracle_join_f32(const float *R, int64_t nR, const float *S, int64_t nS, int d, double T,
                    int mode, int nthreads, uint64_t **out_keys, int64_t *out_count) {
    if (d <= 0 || nR < 0 || nS < 0 || mode < 0 || mode > 2) return -2;
    job_t p;
    memset(&p, 0, sizeof(p));
    p.R = R; p.S = S; p.nR = nR; p.nS = nS; p.d = d; p.T = T; p.mode = mode; p.is_int = 0;
    return run(&p, nthreads, out_keys, out_count);
}

int oracle_join_i16(const int16_t *R, int64_t nR, const int16_t *S, int64_t nS, int d, int64_t T,
                    int mode, int nthreads, uint64_t **out_keys, int64_t *out_count) {
    if (d <= 0 || nR < 0 || nS < 0 || mode < 0 || mode > 2) return -2;
    job_t p;
    memset(&p, 0, sizeof(p));
    p.R = R; p.S = S; p.nR = nR; p.nS = nS; p.d = d; p.Ti = T; p.mode = mode; p.is_int = 1;
    return run(&p, nthreads, out_keys, out_count);
}

void oracle_free(void *p) { free(p); }

/* Sequential-order FP64 squared distances for an explicit list of pairs. */
void oracle_pair_d2_f32(const float *R, const float *S, int d, const int64_t *ii, const int64_t *jj,
                        int64_t n, double *out) {
    for (int64_t p = 0; p < n; ++p) out[p] = seq_d2_f32(R + (size_t)ii[p] * d, S + (size_t)jj[p] * d, d);
}

/* The same for many pairs over `nthreads` threads (contiguous pair ranges), FP32 or int16 rows
 * (int16: exact int64 squared distances). */
typedef struct {
    const void *R, *S;
    int d, is_int;
    const int64_t *ii, *jj;
    int64_t p0, p1;
    void *out;
} pair_job_t;

static void *pair_worker(void *arg) {
    pair_job_t *j = (pair_job_t *)arg;
    const int d = j->d;
    if (!j->is_int) {
        const float *R = (const float *)j->R, *S = (const float *)j->S;
        double *o = (double *)j->out;
        for (int64_t p = j->p0; p < j->p1; ++p) o[p] = seq_d2_f32(R + (size_t)j->ii[p] * d, S + (size_t)j->jj[p] * d, d);
    } else {
        const int16_t *R = (const int16_t *)j->R, *S = (const int16_t *)j->S;
        int64_t *o = (int64_t *)j->out;
        for (int64_t p = j->p0; p < j->p1; ++p) o[p] = exact_d2_i16(R + (size_t)j->ii[p] * d, S + (size_t)j->jj[p] * d, d);
    }
    return NULL;
}

static int pair_run(const void *R, const void *S, int d, int is_int, const int64_t *ii, const int64_t *jj,
                    int64_t n, void *out, int nthreads) {
    if (d <= 0 || n < 0) return -2;
    if (nthreads < 1) nthreads = 1;
    if (nthreads > 256) nthreads = 256;
    if (n < (int64_t)nthreads * 1024) nthreads = 1;
    pair_job_t *jobs = (pair_job_t *)calloc((size_t)nthreads, sizeof(pair_job_t));
    pthread_t *th = (pthread_t *)calloc((size_t)nthreads, sizeof(pthread_t));
    if (!jobs || !th) { free(jobs); free(th); return -1; }
    for (int t = 0; t < nthreads; ++t) {
        pair_job_t j = {R, S, d, is_int, ii, jj, n * t / nthreads, n * (t + 1) / nthreads, out};
        jobs[t] = j;
    }
    for (int t = 1; t < nthreads; ++t) pthread_create(&th[t], NULL, pair_worker, &jobs[t]);
    pair_worker(&jobs[0]);
    for (int t = 1; t < nthreads; ++t) pthread_join(th[t], NULL);
    free(jobs);
    free(th);
    return 0;
}

int oracle_pair_d2_f32_mt(const float *R, const float *S, int d, const int64_t *ii, const int64_t *jj, int64_t n,
                          double *out, int nthreads) {
    return pair_run(R, S, d, 0, ii, jj, n, out, nthreads);
}

int oracle_pair_d2_i16_mt(const int16_t *R, const int16_t *S, int d, const int64_t *ii, const int64_t *jj, int64_t n,
                          int64_t *out, int nthreads) {
    return pair_run(R, S, d, 1, ii, jj, n, out, nthreads);
}

/* Per-row counts of neighbours (row-major scan, no key materialisation); used for large-sample audits. */
int oracle_row_counts_f32(const float *R, int64_t nR, const float *S, int64_t nS, int d, double T,
                          const int64_t *rows, int64_t nrows, int64_t *counts) {
    for (int64_t r = 0; r < nrows; ++r) {
        const float *x = R + (size_t)rows[r] * d;
        int64_t c = 0;
        for (int64_t j = 0; j < nS; ++j) c += seq_d2_f32(x, S + (size_t)j * d, d) <= T;
        counts[r] = c;
    }
    (void)nR;
    return 0;
}

/* Version tag so Python can check it loaded the expected build. */
int oracle_abi_version(void) { return 2; }
