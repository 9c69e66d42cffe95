// Index build: Morton-sorted grid over the highest-variance dimensions or over the top
// principal directions, per-row certificate metadata and low-precision MMA operands, tile
// statistics, and the candidate tile-pair list with its execution chunks.
//
// Reference semantics (restated, not ported):
//  * grid index: GDS-Join's per-dimension cells over NUMINDEXEDDIM variance-ordered
//    dimensions (adapters/gds_g2a/main.cu:419-424 ReorderByDimension, :867-883
//    getLinearID_nDimensions, :891-948 generateNDGridDimensions).  Here the cell
//    coordinates are interleaved into a Morton key and points are radix-sorted by it
//    on the GPU instead of a CPU std::set (main.cu:690-857).
//  * principal-direction layout: the PCA-sorted block layout of the block-feasibility study
//    (tensorjoin_20260908_block_feasibility/src/geometry.py:15-32 projection and layout), built
//    here on the GPU from a sampled covariance and used only to order rows into tiles.
//  * candidate list: the tile-pair schedule of the scripted joins
//    (src/run_g2b_tensorjoin_public.py:211-215, np.triu_indices for self-joins) pruned
//    with conservative block lower bounds, ball and axis-aligned box
//    (tensorjoin_20260908_block_feasibility/src/geometry.py:73-150).
//  * per-row metadata: norms, reconstruction residual bound and low-precision copy
//    (two_gate_campaign_20260908/src/gpu_kernels.py:33-51 half_metadata,
//    g16_gpu_preparation_20260905/src/gpu_preparation.py:13-49).
#include <algorithm>
#include <cmath>

#include "tj_internal.h"

namespace tj {

namespace {

constexpr int kStatBlocks = 1184;   // 8 blocks of 256 threads per SM on 148 SMs

TJ_DEV float load_x(const void* src, int dtype, size_t idx) {
    return dtype == kF32 ? ((const float*)src)[idx] : (float)((const int16_t*)src)[idx];
}

// Per-block partial statistics for every dimension.  Threads are laid out as
// (row group g, dimension k); groups are combined in shared memory in a fixed order.
// Rows rstride * r for r < n (a strided sample of the source when rstride > 1).
__global__ void __launch_bounds__(256) dim_stats_partial(const void* src, int dtype, long long n, long long rstride,
                                                         int d, float* pmin, float* pmax, double* psum, double* psq,
                                                         int blk_base) {
    __shared__ float smn[256], smx[256];
    __shared__ double ss[256], sq[256];
    const int G = d >= 256 ? 1 : 256 / d;
    const long long rows_per = (n + gridDim.x - 1) / gridDim.x;
    const long long r0 = (long long)blockIdx.x * rows_per;
    const long long r1 = min(n, r0 + rows_per);
    for (int kb = 0; kb < d; kb += 256) {
        const int t = threadIdx.x;
        const int g = (d >= 256) ? 0 : t / d;
        const int k = (d >= 256) ? kb + t : t % d;
        float mn = INFINITY, mx = -INFINITY;
        double s = 0.0, q = 0.0;
        if (g < G && k < d) {
            long long r = r0 + g;
            for (; r + 3 * G < r1; r += 4 * G) {   // four independent loads in flight per thread
                float v[4];
#pragma unroll
                for (int u = 0; u < 4; ++u) v[u] = load_x(src, dtype, (size_t)((r + u * G) * rstride) * d + k);
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    mn = fminf(mn, v[u]);
                    mx = fmaxf(mx, v[u]);
                    s += v[u];
                    q += (double)v[u] * v[u];
                }
            }
            for (; r < r1; r += G) {
                const float v = load_x(src, dtype, (size_t)(r * rstride) * d + k);
                mn = fminf(mn, v);
                mx = fmaxf(mx, v);
                s += v;
                q += (double)v * v;
            }
        }
        smn[t] = mn; smx[t] = mx; ss[t] = s; sq[t] = q;
        __syncthreads();
        if (d < 256 && t < d) {
            for (int gg = 1; gg < G; ++gg) {
                const int o = gg * d + t;
                mn = fminf(mn, smn[o]); mx = fmaxf(mx, smx[o]); s += ss[o]; q += sq[o];
            }
        }
        if ((d >= 256 && k < d) || (d < 256 && t < d)) {
            const size_t o = (size_t)(blk_base + blockIdx.x) * d + k;
            pmin[o] = mn;
            pmax[o] = mx;
            psum[o] = s;
            psq[o] = q;
        }
        __syncthreads();
        if (d < 256) break;
    }
}

// Deterministic reduction of the partials (one block per dimension, a fixed-shape tree over the
// partial blocks): variance, range and the centre (per-dimension mean, FP32) used to centre the
// MMA operands.
__global__ void __launch_bounds__(256) dim_reduce(const float* pmin, const float* pmax, const double* psum,
                                                  const double* psq, int nparts, long long ntot, int d,
                                                  float* var_ws, float* lo_ws, float* hi_ws, float* center) {
    __shared__ double ss[256], sq[256];
    __shared__ float smn[256], smx[256];
    const int k = blockIdx.x, t = threadIdx.x;
    float mn = INFINITY, mx = -INFINITY;
    double s = 0.0, q = 0.0;
    for (int b = t; b < nparts; b += blockDim.x) {
        const size_t o = (size_t)b * d + k;
        mn = fminf(mn, pmin[o]);
        mx = fmaxf(mx, pmax[o]);
        s += psum[o];
        q += psq[o];
    }
    ss[t] = s; sq[t] = q; smn[t] = mn; smx[t] = mx;
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
        if (t < w) {
            ss[t] += ss[t + w]; sq[t] += sq[t + w];
            smn[t] = fminf(smn[t], smn[t + w]); smx[t] = fmaxf(smx[t], smx[t + w]);
        }
        __syncthreads();
    }
    if (t == 0) {
        const double mean = ntot ? ss[0] / (double)ntot : 0.0;
        var_ws[k] = ntot ? (float)fmax(0.0, sq[0] / (double)ntot - mean * mean) : 0.f;
        lo_ws[k] = smn[0];
        hi_ws[k] = smx[0];
        center[k] = isfinite(mean) ? (float)mean : 0.f;
    }
}

// Pick the m = min(d, 8) highest-variance dimensions and their quantisation frame (one warp: each
// round a lane-strided scan and a warp arg-max, ties to the lowest dimension).
__global__ void __launch_bounds__(32) frame_pick(int d, const float* var_ws, const float* lo_ws, const float* hi_ws,
                                                 FrameParams* fp) {
    const int lane = threadIdx.x, m = min(d, 8), bits = 32 / m;
    int dims[8];
    for (int t = 0; t < m; ++t) {
        int best = -1;
        float bv = 0.f;
        for (int k = lane; k < d; k += 32) {
            bool used = false;
            for (int u = 0; u < t; ++u) used |= (dims[u] == k);
            if (used) continue;
            if (best < 0 || var_ws[k] > bv) { best = k; bv = var_ws[k]; }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {   // arg-max over lanes; no candidate < any candidate
            const int ob = __shfl_xor_sync(0xffffffffu, best, o);
            const float ov = __shfl_xor_sync(0xffffffffu, bv, o);
            const bool take = ob >= 0 && (best < 0 || ov > bv || (ov == bv && ob < best));
            if (take) { best = ob; bv = ov; }
        }
        dims[t] = best;
    }
    if (lane < m) {
        const int best = dims[lane];
        const float lo = lo_ws[best], hi = hi_ws[best];
        const float range = (isfinite(lo) && isfinite(hi) && hi > lo) ? hi - lo : 1.f;
        fp->dims[lane] = best;
        fp->lo[lane] = isfinite(lo) ? lo : 0.f;
        fp->inv_w[lane] = (float)(1u << bits) / range;
    }
    if (lane == 0) {
        fp->m = m;
        fp->bits = bits;
        fp->pca = 0;
    }
}

TJ_DEV int join_of_row(const long long* rowoff, int njc, long long r) {   // last j with rowoff[j] <= r
    int lo = 0, hi = njc - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (rowoff[mid] <= r) lo = mid; else hi = mid - 1;
    }
    return lo;
}

// Principal-component frame (the PCA-ordered layout): covariance of up to kPcaSamples evenly
// spaced rows of all sources, top m = 8 directions by subspace iteration, cells over the
// projections y_k = (x - c) . v_k quantised on their range over the sampled rows.  The frame only
// decides which rows share a tile; every bound and result stays exact.
constexpr int kCovBlocks = 256;
constexpr long long kPcaSamples = 16384;
constexpr int kPcaRounds = 8;

// Per-block partial covariance (d x d, FP32, rows in a fixed order), d <= kPcaMaxD.
__global__ void __launch_bounds__(256) cov_partial(const void* const* srcs, const long long* offs, int nsrc,
                                                   long long stride, long long nsamp, int d, int dtype,
                                                   const float* center, float* partial) {
    __shared__ float y[32][kPcaMaxD];
    const int dd = d * d;
    float acc[64];
#pragma unroll
    for (int u = 0; u < 64; ++u) acc[u] = 0.f;
    const long long per = (nsamp + gridDim.x - 1) / gridDim.x;
    const long long s0 = (long long)blockIdx.x * per, s1 = min(nsamp, s0 + per);
    for (long long sb = s0; sb < s1; sb += 32) {
        const int rows = (int)min(32ll, s1 - sb);
        for (int e = threadIdx.x; e < 32 * d; e += 256) {
            const int rr = e / d, k = e % d;
            float v = 0.f;
            if (rr < rows) {
                const long long g = (sb + rr) * stride;   // row index over the concatenated sources
                int src = 0;
                while (src + 1 < nsrc && offs[src + 1] <= g) ++src;
                v = load_x(srcs[src], dtype, (size_t)(g - offs[src]) * d + k) - center[k];
                if (!isfinite(v)) v = 0.f;
            }
            y[rr][k] = v;
        }
        __syncthreads();
#pragma unroll
        for (int u = 0; u < 64; ++u) {
            const int e = threadIdx.x + u * 256;
            if (e < dd) {
                const int i = e / d, j = e % d;
                float a = acc[u];
                for (int rr = 0; rr < rows; ++rr) a = fmaf(y[rr][i], y[rr][j], a);
                acc[u] = a;
            }
        }
        __syncthreads();
    }
#pragma unroll
    for (int u = 0; u < 64; ++u) {
        const int e = threadIdx.x + u * 256;
        if (e < dd) partial[(size_t)blockIdx.x * dd + e] = acc[u];
    }
}

// Sum of the per-block partial covariances, in block order (one thread per entry).
__global__ void cov_reduce(const float* partial, int nparts, int dd, float* C) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= dd) return;
    float a = 0.f;
    for (int b = 0; b < nparts; ++b) a += partial[(size_t)b * dd + e];
    C[e] = a;
}

TJ_DEV float warp_sum_f(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Top m = 8 principal directions of C by kPcaRounds rounds of V <- orth(C V) from a fixed start,
// C scaled by 1 / trace(C) first.  Each round: W = C V on all threads, the 8 x 8 Gram matrix
// G = W^T W by the warps, its Cholesky factor G = L L^T (FP64, one thread), then V = W L^-T
// (Cholesky QR).  Should G lose definiteness the previous V is kept: the frame only orders rows.
static_assert(kPcaMaxD == 128, "the Morton projection loads rows in four 32-column blocks");
__global__ void __launch_bounds__(256) pca_frame(const float* Cg, int d, FrameParams* fp) {
    extern __shared__ float sm[];
    __shared__ float G[8][8], Li[8][8];
    __shared__ float s_scale;
    __shared__ int s_ok;
    float* C = sm;                   // [d][d]
    float* V = C + d * d;            // [8][d]
    float* W = V + 8 * d;            // [8][d]
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5, nwarps = blockDim.x >> 5, dd = d * d, m = 8;
    if (t < 32) {
        float tr = 0.f;
        for (int i = lane; i < d; i += 32) tr += Cg[i * d + i];
        tr = warp_sum_f(tr);
        if (lane == 0) s_scale = (tr > 0.f && isfinite(tr)) ? 1.f / tr : 0.f;
    }
    __syncthreads();
    const float scale = s_scale;
    for (int e = t; e < dd; e += blockDim.x) C[e] = Cg[e] * scale;
    for (int e = t; e < m * d; e += blockDim.x) {   // deterministic, linearly independent start
        const int k = e / d, j = e % d;
        V[e] = (j % m == k ? 1.f : 0.f) + 0.001f * (float)((j * 7 + k * 13) % 17);
    }
    __syncthreads();
    for (int it = 0; it < kPcaRounds && scale > 0.f; ++it) {
        for (int e = t; e < m * d; e += blockDim.x) {   // W = C V (C is symmetric: read its columns)
            const int k = e / d, i = e % d;
            float a = 0.f;
            for (int j = 0; j < d; ++j) a = fmaf(C[j * d + i], V[k * d + j], a);
            W[e] = a;
        }
        __syncthreads();
        for (int e = warp; e < 64; e += nwarps) {       // G = W^T W
            const int k = e >> 3, u = e & 7;
            float a = 0.f;
            for (int j = lane; j < d; j += 32) a = fmaf(W[k * d + j], W[u * d + j], a);
            a = warp_sum_f(a);
            if (lane == 0) G[k][u] = a;
        }
        __syncthreads();
        if (t == 0) {   // L = chol(G), Li = L^-1 (lower triangular), FP64
            double L[8][8] = {}, I[8][8] = {};
            bool ok = true;
            for (int k = 0; k < 8 && ok; ++k) {
                for (int u = 0; u <= k; ++u) {
                    double v = 0.5 * ((double)G[k][u] + (double)G[u][k]);
                    for (int q = 0; q < u; ++q) v -= L[k][q] * L[u][q];
                    if (u == k) {
                        if (!(v > 1e-30)) { ok = false; break; }
                        L[k][k] = sqrt(v);
                    } else {
                        L[k][u] = v / L[u][u];
                    }
                }
            }
            if (ok) {
                for (int c = 0; c < 8; ++c) {
                    for (int k = c; k < 8; ++k) {
                        double v = k == c ? 1.0 : 0.0;
                        for (int q = c; q < k; ++q) v -= L[k][q] * I[q][c];
                        I[k][c] = v / L[k][k];
                    }
                }
                for (int k = 0; k < 8; ++k)
                    for (int u = 0; u < 8; ++u) Li[k][u] = (float)I[k][u];
            }
            s_ok = ok ? 1 : 0;
        }
        __syncthreads();
        if (!s_ok) break;
        for (int e = t; e < m * d; e += blockDim.x) {   // V[:, k] = sum_{u <= k} W[:, u] Li[k][u]
            const int k = e / d, i = e % d;
            float a = 0.f;
            for (int u = 0; u <= k; ++u) a = fmaf(W[u * d + i], Li[k][u], a);
            V[e] = a;
        }
        __syncthreads();
    }
    for (int e = t; e < m * d; e += blockDim.x) fp->V[e] = V[e];
    if (t == 0) {
        fp->m = m;
        fp->bits = 32 / m;
        fp->pca = 1;
        for (int k = 0; k < m; ++k) fp->dims[k] = -1;
    }
}

// Projections of one row onto the frame's 8 directions, computed by a whole warp: coalesced reads
// of the row, butterfly sums; every lane returns the full sums.
TJ_DEV void project8_warp(const void* src, int dtype, size_t row, int d, const float* center, const float* V,
                          int lane, float (&y)[8]) {
#pragma unroll
    for (int k = 0; k < 8; ++k) y[k] = 0.f;
    for (int j = lane; j < d; j += 32) {
        const float xv = load_x(src, dtype, row * d + j) - center[j];
#pragma unroll
        for (int k = 0; k < 8; ++k) y[k] = fmaf(xv, V[k * d + j], y[k]);
    }
#pragma unroll
    for (int k = 0; k < 8; ++k) y[k] = warp_sum_f(y[k]);
}

// Range of each projection over the same sampled rows (one warp per row): per-block minima and
// maxima (out[block][k] = min, out[block][8 + k] = max), reduced by pca_range_finish.  Cells span
// the sampled range; rows outside it fall into the edge cells.
__global__ void __launch_bounds__(256) proj_range_partial(const void* const* srcs, const long long* offs, int nsrc,
                                                          long long stride, long long nsamp, int d, int dtype,
                                                          const float* center, const FrameParams* fp, float* out) {
    __shared__ float smn[8][256], smx[8][256];
    float mn[8], mx[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) { mn[k] = INFINITY; mx[k] = -INFINITY; }
    const int lane = threadIdx.x & 31;
    const long long nwarps = (long long)gridDim.x * (blockDim.x / 32);
    for (long long sidx = (long long)blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5); sidx < nsamp;
         sidx += nwarps) {
        const long long g = sidx * stride;
        int src = 0;
        while (src + 1 < nsrc && offs[src + 1] <= g) ++src;
        float y[8];
        project8_warp(srcs[src], dtype, (size_t)(g - offs[src]), d, center, fp->V, lane, y);
#pragma unroll
        for (int k = 0; k < 8; ++k)
            if (isfinite(y[k])) { mn[k] = fminf(mn[k], y[k]); mx[k] = fmaxf(mx[k], y[k]); }
    }
#pragma unroll
    for (int k = 0; k < 8; ++k) { smn[k][threadIdx.x] = mn[k]; smx[k][threadIdx.x] = mx[k]; }
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
        if (threadIdx.x < w) {
#pragma unroll
            for (int k = 0; k < 8; ++k) {
                smn[k][threadIdx.x] = fminf(smn[k][threadIdx.x], smn[k][threadIdx.x + w]);
                smx[k][threadIdx.x] = fmaxf(smx[k][threadIdx.x], smx[k][threadIdx.x + w]);
            }
        }
        __syncthreads();
    }
    if (threadIdx.x < 8) {
        out[blockIdx.x * 16 + threadIdx.x] = smn[threadIdx.x][0];
        out[blockIdx.x * 16 + 8 + threadIdx.x] = smx[threadIdx.x][0];
    }
}

__global__ void pca_range_finish(const float* part, int nparts, FrameParams* fp) {
    const int k = threadIdx.x;
    if (k >= 8) return;
    float lo = INFINITY, hi = -INFINITY;
    for (int b = 0; b < nparts; ++b) {
        lo = fminf(lo, part[b * 16 + k]);
        hi = fmaxf(hi, part[b * 16 + 8 + k]);
    }
    const bool ok = isfinite(lo) && isfinite(hi) && hi > lo;
    fp->lo[k] = ok ? lo : 0.f;
    fp->inv_w[k] = (float)(1u << fp->bits) / (ok ? hi - lo : 1.f);
}

TJ_DEV uint64_t morton_interleave(const unsigned* c, int m, int bits) {
    uint64_t key = 0;
    for (int b = bits - 1; b >= 0; --b)
        for (int t = 0; t < m; ++t) key = (key << 1) | ((c[t] >> b) & 1u);
    return key;
}

// Morton key of the input-dimension cells; with several joins concatenated in one side the join
// index goes above bit 32, so every join's rows stay contiguous after the sort.
__global__ void morton_keys(const void* src, int dtype, long long n, int d, const FrameParams* fpp, uint64_t* keys,
                            uint32_t* vals, const long long* rowoff, int njc) {
    const long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n) return;
    const int m = fpp->m, bits = fpp->bits;
    const unsigned maxc = (1u << bits) - 1u;
    unsigned c[16];
    for (int t = 0; t < m; ++t) {
        const float v = load_x(src, dtype, (size_t)r * d + fpp->dims[t]);
        float q = (v - fpp->lo[t]) * fpp->inv_w[t];
        q = fminf(fmaxf(q, 0.f), (float)maxc);
        c[t] = isfinite(q) ? (unsigned)q : 0u;
    }
    uint64_t key = morton_interleave(c, m, bits);
    if (njc > 1) key |= (uint64_t)join_of_row(rowoff, njc, r) << 32;
    keys[r] = key;
    vals[r] = (uint32_t)r;
}

// Morton key of the principal-direction cells.  Each warp projects its 32 rows four at a time:
// all of a group's row loads issue together (coalesced, four 32-column blocks), then one
// reduce-scatter over the 4 x 8 partial sums (31 shuffles; lane L ends with row L / 8, direction
// L % 8), routed through shared memory to the row's lane.  Launched with 256 threads.
__global__ void __launch_bounds__(256, 3) morton_keys_pca(const void* src, int dtype, long long n, int d,
                                                          const FrameParams* fpp, uint64_t* keys, uint32_t* vals,
                                                          const long long* rowoff, int njc, const float* center) {
    __shared__ float ybuf[8][32][9];
    const long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const long long w0 = r - lane;
    for (int q0 = 0; q0 < 32 && w0 + q0 < n; q0 += 4) {   // warp-uniform bound: every lane shuffles
        float a[32];   // a[u * 8 + t]: row q0 + u, direction t
#pragma unroll
        for (int e = 0; e < 32; ++e) a[e] = 0.f;
        float xv[4][4];   // [column block jj][row u]
#pragma unroll
        for (int jj = 0; jj < kPcaMaxD / 32; ++jj) {
            const int j = lane + 32 * jj;
#pragma unroll
            for (int u = 0; u < 4; ++u)
                xv[jj][u] = (j < d && w0 + q0 + u < n) ? load_x(src, dtype, (size_t)(w0 + q0 + u) * d + j) : 0.f;
        }
#pragma unroll
        for (int jj = 0; jj < kPcaMaxD / 32; ++jj) {
            const int j = lane + 32 * jj;
            if (j < d) {
                const float cj = center[j];
#pragma unroll
                for (int t = 0; t < 8; ++t) {
                    const float v = fpp->V[t * d + j];
#pragma unroll
                    for (int u = 0; u < 4; ++u) a[u * 8 + t] = fmaf(xv[jj][u] - cj, v, a[u * 8 + t]);
                }
            }
        }
        // reduce-scatter: at width h, lanes with bit h set keep the upper half of the entries
#pragma unroll
        for (int h = 16; h >= 1; h >>= 1) {
            const bool up = (lane & h) != 0;
#pragma unroll
            for (int e = 0; e < h; ++e) {
                const float send = up ? a[e] : a[e + h];
                const float keep = up ? a[e + h] : a[e];
                a[e] = keep + __shfl_xor_sync(0xffffffffu, send, h);
            }
        }
        ybuf[wib][q0 + (lane >> 3)][lane & 7] = a[0];
    }
    __syncwarp();
    if (r >= n) return;
    const int bits = fpp->bits;
    const unsigned maxc = (1u << bits) - 1u;
    unsigned c[8];
#pragma unroll
    for (int t = 0; t < 8; ++t) {
        float q = (ybuf[wib][lane][t] - fpp->lo[t]) * fpp->inv_w[t];
        q = fminf(fmaxf(q, 0.f), (float)maxc);
        c[t] = isfinite(q) ? (unsigned)q : 0u;
    }
    uint64_t key = morton_interleave(c, 8, bits);
    if (njc > 1) key |= (uint64_t)join_of_row(rowoff, njc, r) << 32;
    keys[r] = key;
    vals[r] = (uint32_t)r;
}

__global__ void perm_local_kernel(const uint64_t* keys, const uint32_t* perm, const long long* rowoff, long long n,
                                  uint32_t* out) {
    const long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (r < n) out[r] = (uint32_t)((long long)perm[r] - rowoff[keys[r] >> 32]);
}

// int14 sides: the rows of every 128-row tile put in order of their exact squared norm (ties by
// position).  The int8-limb screens test 8 columns of an S tile at a time against the smallest norm of
// the 8; with norms rising along the tile that bound stays close to every column's own.  A tile keeps
// its rows (only their order inside it changes), so candidate tile pairs and results are unchanged.
// Block per tile, a warp per row for the norms, rank by counting in shared memory.
__global__ void __launch_bounds__(128) order_tile_rows_by_norm(const void* src, int dtype, long long n, int d,
                                                              uint32_t* perm) {
    __shared__ long long key[128];
    __shared__ uint32_t pv[128];
    const long long r0 = (long long)blockIdx.x * 128;
    const int nv = (int)min(128ll, n - r0);
    const unsigned warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int i = (int)warp; i < nv; i += 4) {
        const uint32_t o = perm[r0 + i];
        long long s = 0;
        for (int k = (int)lane; k < d; k += 32) {
            const long long q = (long long)load_x(src, dtype, (size_t)o * d + k);
            s += q * q;
        }
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
        if (lane == 0) {
            key[i] = s;
            pv[i] = o;
        }
    }
    __syncthreads();
    const int t = (int)threadIdx.x;
    if (t < nv) {
        const long long kt = key[t];
        int rank = 0;
        for (int u = 0; u < nv; ++u) {
            const long long ku = key[u];
            rank += (ku < kt || (ku == kt && u < t)) ? 1 : 0;
        }
        perm[r0 + rank] = pv[t];
    }
}

// Concatenate many row-major matrices (one per join) into one: row r of the output comes from the
// source whose row range contains r.
__global__ void gather_rows_kernel(const void* const* srcs, const long long* rowoff, int nsrc, long long nrows,
                                   int row_bytes, uint8_t* dst) {
    const long long r = (long long)blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5);
    if (r >= nrows) return;
    const int j = join_of_row(rowoff, nsrc, r);
    const uint8_t* src = (const uint8_t*)srcs[j] + (size_t)(r - rowoff[j]) * row_bytes;
    uint8_t* out = dst + (size_t)r * row_bytes;
    if ((row_bytes & 3) == 0 && (((uintptr_t)src | (uintptr_t)out) & 3) == 0) {
        for (int b = (threadIdx.x & 31) * 4; b < row_bytes; b += 128)
            *(uint32_t*)(out + b) = *(const uint32_t*)(src + b);
    } else {
        for (int b = threadIdx.x & 31; b < row_bytes; b += 32) out[b] = src[b];
    }
}

// Round to the 16-bit operand format; returns the rounded value as FP32 and its bit pattern.
template <int kFmt>   // 1 = bf16, 0 = fp16
TJ_DEV float round16(float v, uint16_t& bits) {
    if (kFmt == 1) {
        const __nv_bfloat16 h = __float2bfloat16_rn(v);
        bits = __bfloat16_as_ushort(h);
        return __bfloat162float(h);
    }
    const __half h = __float2half_rn(v);
    bits = __half_as_ushort(h);
    return __half2float(h);
}

// Two values rounded to the 16-bit format at once (one packed conversion): returns the packed word
// (a in the low half, b in the high half, the operand layout) and the two rounded values.  The
// same round-to-nearest-even as round16 per value.
template <int kFmt>
TJ_DEV uint32_t round16x2(float a, float b, float& ra, float& rb) {
    uint32_t w;
    if (kFmt == 1) {
        const __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
        w = *reinterpret_cast<const uint32_t*>(&h);
        ra = __uint_as_float(w << 16);
        rb = __uint_as_float(w & 0xFFFF0000u);
    } else {
        const __half2 h = __floats2half2_rn(a, b);
        w = *reinterpret_cast<const uint32_t*>(&h);
        ra = __low2float(h);
        rb = __high2float(h);
    }
    return w;
}

// One group of kL lanes per sorted row (a warp for wide rows, 4 or 8 lanes for rows of at most
// 16 or 32 elements): operand conversion and certificate metadata.
//   plain:      FP32 copy in sorted order, ||x||^2.
//   16-bit:     x' = x - c (c the per-dimension centre; distances are translation invariant),
//               z_hi = round16(x'), and with kSplit also z_lo = round16(x' - z_hi); operand row
//               [z_hi (kpad) | z_lo (kpad)].  Metadata: A = ||x'||^2 (FP64), Y >= ||x'||,
//               Z >= ||z_hi + z_lo||, Zl >= ||z_lo||, E >= ||x' - z_hi - z_lo||.
//   int8 limbs: q = 128 h + l for int14 input, exact integer ||q||^2.
template <int kScreen, int kSplit, int kL>   // kL lanes per row (4, 8 or 32): 32 / kL rows per warp
__global__ void prep_rows(const void* src, int dtype, long long n, int d, int kpad, long long rows_pad,
                          const uint32_t* perm, const float* center, uint16_t* op, int8_t* op8, float* xs,
                          double* nrm2, float* nrm2f, float* zn, float* en, float* yn, float* zl, long long* inorm,
                          unsigned long long* status) {
    const long long r = ((long long)blockIdx.x * blockDim.x + threadIdx.x) / kL;
    const unsigned sub = threadIdx.x % kL;
    const bool live = r < rows_pad;          // lanes past the end still take part in the shuffles
    const bool real = live && r < n;
    const size_t orig = real ? (size_t)perm[r] : 0;
    double sx = 0.0, sz = 0.0, se = 0.0, sl = 0.0;
    long long sq = 0;
    unsigned flags = 0;   // 1: bad input, 2: FP16 range
    const int opw = kSplit ? 2 * kpad : kpad;
    constexpr int kU = 4;   // elements per lane whose loads are issued together
    for (int k0 = sub; k0 < kpad && live; k0 += kU * kL) {
      float xv[kU];
#pragma unroll
      for (int u = 0; u < kU; ++u) {
          const int k = k0 + u * kL;
          xv[u] = (real && k < d) ? load_x(src, dtype, orig * d + k) : 0.f;
      }
#pragma unroll
      for (int u = 0; u < kU; ++u) {
        const int k = k0 + u * kL;
        if (k >= kpad) break;
        float x = xv[u];
        if (!isfinite(x)) { flags |= 1u; x = 0.f; }
        if (kScreen == kScreenPlain) {
            if (k < d) xs[(size_t)r * d + k] = x;
            sx += (double)x * x;
        } else if (kScreen == kScreenInt8Limb) {   // q = 128 h + l, h = floor((q + 64) / 128)
            const int q = (int)x;
            if (q < -8192 || q > 8191) flags |= 1u;
            const int h = (q + 64 + 8192) / 128 - 64;
            const int l = q - 128 * h;
            op8[(size_t)r * (2 * kpad) + k] = (int8_t)h;
            op8[(size_t)r * (2 * kpad) + kpad + k] = (int8_t)l;
            sq += (long long)q * q;
            sx += (double)x * x;
            sz += (double)(h * h);   // |h|^2 and |l|^2 exactly (small integers): zn, zl bound the limb norms
            sl += (double)(l * l);
        } else {
            constexpr int kFmt = (kScreen == kScreenBF16 || kScreen == kScreenBF16X3) ? 1 : 0;
            const double xc = (k < d && real) ? (double)x - (double)center[k] : 0.0;
            const float xf = (float)xc;
            if (kFmt == 0 && fabsf(xf) > 65504.f) flags |= 2u;
            uint16_t bh = 0, bl = 0;
            const float zh = round16<kFmt>(xf, bh);
            double z = (double)zh;
            if (kSplit) {
                const float zlo = round16<kFmt>((float)(xc - (double)zh), bl);
                z += (double)zlo;
                sl += (double)zlo * zlo;
                op[(size_t)r * opw + kpad + k] = bl;
            }
            op[(size_t)r * opw + k] = bh;
            const double ed = xc - z;
            sx += xc * xc;
            sz += z * z;
            se += ed * ed;
        }
      }
    }
#pragma unroll
    for (int o = kL / 2; o > 0; o >>= 1) {
        sx += __shfl_xor_sync(0xffffffffu, sx, o);
        sz += __shfl_xor_sync(0xffffffffu, sz, o);
        se += __shfl_xor_sync(0xffffffffu, se, o);
        sl += __shfl_xor_sync(0xffffffffu, sl, o);
        sq += __shfl_xor_sync(0xffffffffu, sq, o);
        flags |= __shfl_xor_sync(0xffffffffu, flags, o);
    }
    // FP64 sums of d non-negative squares (each rounded once): relative error <= (d+2) 2^-53;
    // x - c may round once more (2^-53 relative), absorbed by the extra 2^-50 terms.
    // The four norm bounds of a row are taken by its first four lanes, one square root each in the
    // same instruction stream (every lane computes one; kL >= 4), instead of four in a row on one lane.
    static_assert(kL >= 4, "four lanes per row take the four norm bounds");
    const double g = (double)(d + 4) * 0x1p-53;
    const double up = (1.0 + 2.0 * g) * (1.0 + 0x1p-50);
    const unsigned task = sub & 3u;   // 0: |x - c|, 1: |w|, 2: |x - c - w|, 3: |w_lo|
    const double v = task == 0 ? sx : task == 1 ? sz : task == 2 ? se : sl;
    double rt = sqrt(v * up) * (1.0 + 0x1p-50);
    const double ynorm = __shfl_sync(0xffffffffu, rt, (int)((threadIdx.x & 31u) & ~(unsigned)(kL - 1)));
    if (task == 2) rt += 0x1p-50 * ynorm;
    if (live && sub < 4) {
        float* dst = task == 0 ? yn : task == 1 ? zn : task == 2 ? en : zl;
        dst[r] = f32_up(rt);
    }
    if (sub == 0 && live) {
        if ((flags & 1u) && real) atomicOr(status, (unsigned long long)kStatusBadInput);
        if ((flags & 2u) && real) atomicOr(status, (unsigned long long)kStatusFp16Range);
        if (real && sx > 0x1p100) atomicOr(status, (unsigned long long)kStatusBadInput);
        nrm2[r] = sx;
        nrm2f[r] = __double2float_rn(sx);
        if (inorm) inorm[r] = sq;
    }
}

// Tile statistics: one block per tile; kL lanes per row (4, 8 or 32), 256 / kL rows at a time.
template <int kL>
__global__ void __launch_bounds__(256) tile_stats_kernel(const void* src, int dtype, long long n, int d, int tile,
                                                         int ntiles, const uint32_t* perm, const double* nrm2,
                                                         const float* nrm2f, const float* zn, const float* en,
                                                         const float* yn, const float* zl, float* ctrT, float* loT,
                                                         float* hiT, float* rad, float* maxZ, float* maxE,
                                                         float* maxY, float* maxB, float* beta, float* maxZl,
                                                         uint32_t* nvalid, uint32_t* row0, const uint32_t* row0_in,
                                                         const uint32_t* nvalid_in, int warp_rows) {
    extern __shared__ float s_ctr[];   // [d]
    __shared__ float red[6][256];
    const int t = blockIdx.x;
    const bool tabled = row0_in != nullptr;   // batched sides: tiles never span two joins
    const long long r0 = tabled ? (long long)row0_in[t] : (long long)t * tile;
    const int nv = tabled ? (int)nvalid_in[t] : (int)min((long long)tile, n - r0);
    const double g = (double)(d + 2) * 0x1p-53;
    // per-dimension centroid and bounding box
    const unsigned lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    constexpr int kNG = 256 / kL;                   // row groups per block
    const int grp = threadIdx.x / kL, sub = threadIdx.x % kL;
    if (warp_rows) {
        // group q reads rows q, q + kNG, ... (coalesced across dimensions); per-group partials in
        // shared memory, combined over the groups in a fixed order
        double* psum = (double*)(s_ctr + ((d + 1) & ~1));   // [kNG][d]
        float* pmin = (float*)(psum + kNG * d);             // [kNG][d]
        float* pmax = pmin + kNG * d;                       // [kNG][d]
        for (int k = sub; k < d; k += kL) {
            psum[grp * d + k] = 0.0;
            pmin[grp * d + k] = INFINITY;
            pmax[grp * d + k] = -INFINITY;
        }
        constexpr int kU = 8;   // rows of a group whose loads are issued together
        for (int i = grp; i < nv; i += kU * kNG) {
            size_t base[kU];
#pragma unroll
            for (int u = 0; u < kU; ++u) {
                const int ii = i + u * kNG;
                base[u] = ii < nv ? (size_t)perm[r0 + ii] * d : 0;
            }
            for (int k = sub; k < d; k += kL) {
                float v[kU];
#pragma unroll
                for (int u = 0; u < kU; ++u) v[u] = i + u * kNG < nv ? load_x(src, dtype, base[u] + k) : 0.f;
                double sm = psum[grp * d + k];
                float mn = pmin[grp * d + k], mx = pmax[grp * d + k];
#pragma unroll
                for (int u = 0; u < kU; ++u) {
                    if (i + u * kNG < nv) {
                        sm += v[u];
                        mn = fminf(mn, v[u]);
                        mx = fmaxf(mx, v[u]);
                    }
                }
                psum[grp * d + k] = sm;
                pmin[grp * d + k] = mn;
                pmax[grp * d + k] = mx;
            }
        }
        __syncthreads();
        for (int k = threadIdx.x; k < d; k += blockDim.x) {
            double sm = 0.0;
            float mn = INFINITY, mx = -INFINITY;
            for (int w = 0; w < kNG; ++w) {
                sm += psum[w * d + k];
                mn = fminf(mn, pmin[w * d + k]);
                mx = fmaxf(mx, pmax[w * d + k]);
            }
            const float c = (float)(sm / (double)max(nv, 1));
            s_ctr[k] = c;
            ctrT[(size_t)k * ntiles + t] = c;
            loT[(size_t)k * ntiles + t] = mn;
            hiT[(size_t)k * ntiles + t] = mx;
        }
    } else {
        for (int k = threadIdx.x; k < d; k += blockDim.x) {
            double sm = 0.0;
            float mn = INFINITY, mx = -INFINITY;
            for (int i = 0; i < nv; ++i) {
                const float v = load_x(src, dtype, (size_t)perm[r0 + i] * d + k);
                sm += v;
                mn = fminf(mn, v);
                mx = fmaxf(mx, v);
            }
            const float c = (float)(sm / (double)max(nv, 1));
            s_ctr[k] = c;
            ctrT[(size_t)k * ntiles + t] = c;
            loT[(size_t)k * ntiles + t] = mn;
            hiT[(size_t)k * ntiles + t] = mx;
        }
    }
    __syncthreads();
    // radius: kL lanes per row, exact FP64 differences against the FP32 centroid; the row loop is
    // uniform across each warp so that every lane takes part in the shuffles
    double rmax = 0.0;
    constexpr int kRU = 4;   // rows per lane group whose loads are issued together
    for (int i0 = warp * (32 / kL); i0 < nv; i0 += kRU * kNG) {
        double s[kRU];
        size_t base[kRU];
        bool ok[kRU];
#pragma unroll
        for (int u = 0; u < kRU; ++u) {
            const int i = i0 + u * kNG + (int)(lane / kL);
            ok[u] = i < nv;
            base[u] = ok[u] ? (size_t)perm[r0 + i] * d : 0;
            s[u] = 0.0;
        }
        for (int k = sub; k < d; k += kL) {
            float v[kRU];
#pragma unroll
            for (int u = 0; u < kRU; ++u) v[u] = ok[u] ? load_x(src, dtype, base[u] + k) : 0.f;
            const double c = (double)s_ctr[k];
#pragma unroll
            for (int u = 0; u < kRU; ++u) {
                const double df = (double)v[u] - c;
                if (ok[u]) s[u] += df * df;
            }
        }
#pragma unroll
        for (int u = 0; u < kRU; ++u) {
#pragma unroll
            for (int o = kL / 2; o > 0; o >>= 1) s[u] += __shfl_xor_sync(0xffffffffu, s[u], o);
            rmax = fmax(rmax, s[u]);
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) rmax = fmax(rmax, __shfl_xor_sync(0xffffffffu, rmax, o));
    // row-bound maxima
    float mz = 0.f, me = 0.f, my = 0.f, mb = 0.f, mbeta = 0.f, mzl = 0.f;
    for (int i = threadIdx.x; i < nv; i += blockDim.x) {
        const long long r = r0 + i;
        mz = fmaxf(mz, zn[r]);
        me = fmaxf(me, en[r]);
        my = fmaxf(my, yn[r]);
        mb = fmaxf(mb, nrm2f[r]);
        mzl = fmaxf(mzl, zl[r]);
        const double bt = fabs((double)nrm2f[r] - nrm2[r]) + 2.0 * g * nrm2[r];
        mbeta = fmaxf(mbeta, f32_up(bt * (1.0 + 0x1p-40)));
    }
    red[0][threadIdx.x] = mz;
    red[1][threadIdx.x] = me;
    red[2][threadIdx.x] = my;
    red[3][threadIdx.x] = mb;
    red[4][threadIdx.x] = mbeta;
    red[5][threadIdx.x] = mzl;
    __shared__ double rr[8];
    if (lane == 0) rr[warp] = rmax;
    __syncthreads();
    for (int s = 128; s > 0; s >>= 1) {
        if (threadIdx.x < s)
            for (int q = 0; q < 6; ++q) red[q][threadIdx.x] = fmaxf(red[q][threadIdx.x], red[q][threadIdx.x + s]);
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        double m = 0.0;
        for (int w = 0; w < 8; ++w) m = fmax(m, rr[w]);
        // FP64 sum of d squares of exact differences: relative error <= g; sqrt correctly rounded
        rad[t] = f32_up(sqrt(m * (1.0 + 2.0 * g)) * (1.0 + 0x1p-50));
        maxZ[t] = red[0][0];
        maxE[t] = red[1][0];
        maxY[t] = red[2][0];
        maxB[t] = red[3][0];
        beta[t] = red[4][0];
        maxZl[t] = red[5][0];
        if (!tabled) {
            nvalid[t] = (uint32_t)max(nv, 0);
            row0[t] = (uint32_t)r0;
        }
    }
}

// Outputs of the fused kernel for one tile granularity.
struct TileOut {
    float *ctrT, *loT, *hiT, *rad, *maxZ, *maxE, *maxY, *maxB, *beta, *maxZl;
    uint32_t *nvalid, *row0;
    int ntiles;
};

// Constants of the fused operand pass for rows of d elements (see prep_tiles_kernel).
struct PrepBounds {
    double up64;     // (1 + 2 (d + 4) 2^-53)(1 + 2^-50): A's relative error and its product's rounding
    float up32;      // 1 + (d + 16) 2^-23: FP32 sums of d squares (exact in FP32 for d <= 128)
    float slack32;   // d 2^-140: the products that underflow
    double gb;       // (d + 2) 2^-53: beta = |nrm2f - nrm2| + 2 gb nrm2
    TJ_DEV explicit PrepBounds(int d)
        : up64((1.0 + 2.0 * (double)(d + 4) * 0x1p-53) * (1.0 + 0x1p-50)),
          up32(1.f + (float)(d + 16) * 0x1p-23f),
          slack32((float)d * 0x1p-140f),
          gb((double)(d + 2) * 0x1p-53) {}
};

// One sorted row of the fused operand pass: a group of kL lanes holds the row, kE consecutive elements
// per lane (k0 = kE sub).  Writes the row's operands (when rv), its norms and bounds (its first four
// lanes, one bound each), and adds the row to this lane's centroid / box partials and bound maxima.
// Every lane of the warp calls it (the row reduction is a shuffle tree inside the group).
template <int kScreen, int kSplit, int kE, int kL>
TJ_DEV void prep_row(const float (&xa)[kE], const float (&cf)[kE], const double (&cdv)[kE], bool rv, long long r,
                     int k0, int d, unsigned sub, unsigned lane, const PrepBounds& pb, uint16_t* op, double* nrm2,
                     float* nrm2f, float* zn, float* en, float* yn, float* zl, float (&ps)[kE], float (&pl)[kE],
                     float (&ph)[kE], float& mtask, float& mb, float& mbeta, unsigned& flags) {
    constexpr int kFmt = (kScreen == kScreenBF16 || kScreen == kScreenBF16X3) ? 1 : 0;
    constexpr int kPad = kE * kL;
    constexpr int opw = kSplit ? 2 * kPad : kPad;
    double sx = 0.0;
    float sz = 0.f, se = 0.f, sl = 0.f;
    uint32_t hw[kE / 2], lw[kE / 2];
    // element pairs (one packed 16-bit conversion per pair and part); every sum still runs over the
    // elements in order
#pragma unroll
    for (int q = 0; q < kE; q += 2) {
        float sd[2], zh[2], d1[2];
#pragma unroll
        for (int e = 0; e < 2; ++e) {
            sd[e] = xa[q + e] - cf[q + e];   // fl32(x'): |x' - sd| <= 2^-24 |x'| per element
            const double xd = (double)xa[q + e] - cdv[q + e];
            sx = fma(xd, xd, sx);
            if (kFmt == 0 && fabsf(sd[e]) > 65504.f) flags |= 2u;
        }
        hw[q / 2] = round16x2<kFmt>(sd[0], sd[1], zh[0], zh[1]);
        d1[0] = sd[0] - zh[0];   // exact (zh is sd rounded to 8 or 11 bits)
        d1[1] = sd[1] - zh[1];
        if (kSplit) {
            float zlo[2];
            lw[q / 2] = round16x2<kFmt>(d1[0], d1[1], zlo[0], zlo[1]);
#pragma unroll
            for (int e = 0; e < 2; ++e) {
                const float ed = d1[e] - zlo[e];   // exact: sd - z_hi - z_lo
                const float z = zh[e] + zlo[e];
                sz = fmaf(z, z, sz);
                se = fmaf(ed, ed, se);
                sl = fmaf(zlo[e], zlo[e], sl);
            }
        } else {
            lw[q / 2] = 0u;
#pragma unroll
            for (int e = 0; e < 2; ++e) {
                sz = fmaf(zh[e], zh[e], sz);
                se = fmaf(d1[e], d1[e], se);   // d1 = sd - z_hi exactly
            }
        }
#pragma unroll
        for (int e = 0; e < 2; ++e) {
            if (rv && k0 + q + e < d) {
                ps[q + e] += xa[q + e];
                pl[q + e] = fminf(pl[q + e], xa[q + e]);
                ph[q + e] = fmaxf(ph[q + e], xa[q + e]);
            }
        }
    }
    if (rv) {
#pragma unroll
        for (int v = 0; v < kE / 4; ++v) {
            *reinterpret_cast<uint2*>(op + (size_t)r * opw + k0 + 4 * v) = make_uint2(hw[2 * v], hw[2 * v + 1]);
            if (kSplit)
                *reinterpret_cast<uint2*>(op + (size_t)r * opw + kPad + k0 + 4 * v) =
                    make_uint2(lw[2 * v], lw[2 * v + 1]);
        }
    }
#pragma unroll
    for (int o = kL / 2; o > 0; o >>= 1) {
        sx += __shfl_xor_sync(0xffffffffu, sx, o);
        sz += __shfl_xor_sync(0xffffffffu, sz, o);
        se += __shfl_xor_sync(0xffffffffu, se, o);
        if (kSplit) sl += __shfl_xor_sync(0xffffffffu, sl, o);
    }
    // the four bounds of the row are taken by its first four lanes, one square root each
    const unsigned task = sub & 3u;   // 0: |x - c|, 1: |z|, 2: |x - c - z|, 3: |z_lo|
    float rt;
    if (task == 0) {
        rt = __fsqrt_ru(__double2float_ru(sx * pb.up64));
    } else {
        const float v32 = task == 1 ? sz : task == 2 ? se : sl;
        rt = (task == 3 && !kSplit) ? 0.f : __fsqrt_ru(__fmul_ru(__fadd_ru(v32, pb.slack32), pb.up32));
    }
    // E also covers x' - sd (at most 2^-24 |x'| per element, so 2^-24 Y in norm; 2^-23 Y taken)
    const float ynorm = __shfl_sync(0xffffffffu, rt, (int)(lane & ~(unsigned)(kL - 1)));
    if (task == 2) rt = __fadd_ru(rt, __fmul_ru(0x1p-23f, ynorm));
    if (rv && sub < 4) {
        float* dst = task == 0 ? yn : task == 1 ? zn : task == 2 ? en : zl;
        dst[r] = rt;
        mtask = fmaxf(mtask, rt);
    }
    if (rv && sub == 0) {
        if (!(sx <= 0x1p100)) flags |= 1u;   // also NaN / Inf anywhere in the row
        const float sf = __double2float_rn(sx);
        nrm2[r] = sx;
        nrm2f[r] = sf;
        mb = fmaxf(mb, sf);
        const double bt = fabs((double)sf - sx) + 2.0 * pb.gb * sx;
        mbeta = fmaxf(mbeta, f32_up(bt * (1.0 + 0x1p-40)));
    }
}

// Operand preparation and tile statistics in one pass, for 16-bit screens over FP32 rows with
// d % 4 == 0 and kpad = kE kL <= 128 (one block of 256 threads per tile of 128 or 256 sorted rows;
// kL lanes per row, each lane kE consecutive elements).  Every gathered row is read from HBM once:
// the row's operands, norms and bounds, and the tile's centroid and box partials come from that
// read; the radius pass reads the tile again while it is still in L2.  With kHalves the statistics
// of the two 128-row halves of a 256-row tile are written as well (tile t, half h -> entry 2 t + h
// of H).  Partials are combined across the row groups of a warp by shuffles and across the eight
// warps in shared memory.
//
// Arithmetic.  The operands split s = fl32(x - c), which differs from x' = x - c by at most
// 2^-24 |x'| per element (a difference that is subnormal is exact): z_hi = round16(s), and with the
// split z_lo = round16(s - z_hi); s - z_hi and s - z_hi - z_lo are exact in FP32.  So
// ||x' - z|| <= ||s - z|| + 2^-24 ||x'||, and E adds 2^-23 Y to the bound of ||s - z||.
// A = ||x'||^2 stays an FP64 sum of the exact x' (its relative error enters the certificate).
// Z >= ||z_hi + z_lo||, ||s - z||, Zl >= ||z_lo|| and the tile radius are FP32 sums of squares made
// rigorous upper bounds: each term is exact or rounded once (relative 2^-24; additions are exact in
// the subnormal range, a product that underflows errs by at most 2^-150), a chain of m <= d + 5
// roundings errs by at most gamma_m, so  true <= (S + d 2^-140) (1 + (d + 16) 2^-23);  that widening
// and the square root are taken with upward rounding (FP32 .ru operations), as is
// Y = sqrt(A (1 + 2 g)).  A non-finite element makes A non-finite, which flags the row.  The
// centroid needs no accuracy (the radius is measured from the value written).
template <int kScreen, int kSplit, int kE, int kL, bool kHalves>
__global__ void __launch_bounds__(256, 3) prep_tiles_kernel(const float* __restrict__ src, long long n, int d, int tile,
                                                         const uint32_t* __restrict__ perm,
                                                         const float* __restrict__ center,
                                                         const uint32_t* row0_in, const uint32_t* nvalid_in,
                                                         uint16_t* op, double* nrm2, float* nrm2f, float* zn,
                                                         float* en, float* yn, float* zl, TileOut T, TileOut H,
                                                         unsigned long long* status) {
    constexpr int kPad = kE * kL;
    constexpr int kNG = 256 / kL;              // row groups per block
    constexpr int kRows = 128 / kNG;           // rows of one group in one 128-row half
    constexpr int kU = kRows < 2 ? kRows : 2;  // rows whose loads are issued together
    constexpr int kV = kE / 4;                 // float4 loads per lane and row
    static_assert(kE % 4 == 0 && kPad <= 128 && kL >= 4 && kL <= 32, "fused preparation shape");
    __shared__ float wsum[2][8][kPad], wmin[2][8][kPad], wmax[2][8][kPad];   // [half][warp][element]
    __shared__ float wrow[2][6][8];          // [half][bound][warp] row-bound maxima
    __shared__ float wrad[3][8];             // [tile, half 0, half 1][warp] radius-sum maxima
    __shared__ float cs[3][kPad];            // centroids: tile, half 0, half 1
    const int t = blockIdx.x;
    const bool tabled = row0_in != nullptr;
    const long long r0 = tabled ? (long long)row0_in[t] : (long long)t * tile;
    const int nv = tabled ? (int)nvalid_in[t] : (int)min((long long)tile, n - r0);
    const int halves = tile == 256 ? 2 : 1;
    const int grp = threadIdx.x / kL, sub = threadIdx.x % kL;
    const unsigned lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int k0 = kE * sub;
    const bool kin = k0 < d;                   // d % 4 == 0: a float4 is wholly inside or outside
    float cf[kE];
    double cdv[kE];
#pragma unroll
    for (int q = 0; q < kE; ++q) {
        cf[q] = (k0 + q < d) ? center[k0 + q] : 0.f;
        cdv[q] = (double)cf[q];
    }
    const PrepBounds pb(d);
    const float up32 = pb.up32, slack32 = pb.slack32;
    unsigned flags = 0;

    for (int h = 0; h < halves; ++h) {
        const int hb = h * 128;
        float ps[kE], pl[kE], ph[kE];
#pragma unroll
        for (int q = 0; q < kE; ++q) { ps[q] = 0.f; pl[q] = INFINITY; ph[q] = -INFINITY; }
        float mtask = 0.f, mb = 0.f, mbeta = 0.f;   // lanes 0-3 of a group: max of their bound; lane 0: B, beta
        if (hb < nv) {   // uniform across the block
            for (int m0 = 0; m0 < kRows; m0 += kU) {
                float4 xv[kU][kV];
                int ii[kU];
#pragma unroll
                for (int u = 0; u < kU; ++u) {
                    ii[u] = hb + grp + (m0 + u) * kNG;
                    const bool ld = ii[u] < nv && kin;
                    const float4* rowp = ld ? reinterpret_cast<const float4*>(
                                                  src + (size_t)perm[r0 + ii[u]] * (size_t)d + k0)
                                            : nullptr;
#pragma unroll
                    for (int v = 0; v < kV; ++v)
                        xv[u][v] = (ld && k0 + 4 * v < d) ? __ldg(rowp + v) : make_float4(0.f, 0.f, 0.f, 0.f);
                }
#pragma unroll
                for (int u = 0; u < kU; ++u) {
                    float xa[kE];
#pragma unroll
                    for (int q = 0; q < kE; ++q) {
                        const float4 f4 = xv[u][q / 4];
                        xa[q] = (q & 3) == 0 ? f4.x : (q & 3) == 1 ? f4.y : (q & 3) == 2 ? f4.z : f4.w;
                    }
                    prep_row<kScreen, kSplit, kE, kL>(xa, cf, cdv, ii[u] < nv, r0 + ii[u], k0, d, (unsigned)sub, lane,
                                                      pb, op, nrm2, nrm2f, zn, en, yn, zl, ps, pl, ph, mtask, mb,
                                                      mbeta, flags);
                }
            }
        }
        // combine over the row groups of this warp (lanes with the same sub), then per warp to shared
#pragma unroll
        for (int o = kL; o < 32; o <<= 1) {
#pragma unroll
            for (int q = 0; q < kE; ++q) {
                ps[q] += __shfl_xor_sync(0xffffffffu, ps[q], o);
                pl[q] = fminf(pl[q], __shfl_xor_sync(0xffffffffu, pl[q], o));
                ph[q] = fmaxf(ph[q], __shfl_xor_sync(0xffffffffu, ph[q], o));
            }
            mtask = fmaxf(mtask, __shfl_xor_sync(0xffffffffu, mtask, o));
            mb = fmaxf(mb, __shfl_xor_sync(0xffffffffu, mb, o));
            mbeta = fmaxf(mbeta, __shfl_xor_sync(0xffffffffu, mbeta, o));
        }
        if ((int)lane < kL) {   // the warp's first group holds the warp's combined partials
#pragma unroll
            for (int q = 0; q < kE; ++q) {
                wsum[h][warp][k0 + q] = ps[q];
                wmin[h][warp][k0 + q] = pl[q];
                wmax[h][warp][k0 + q] = ph[q];
            }
            if (sub < 4) wrow[h][sub][warp] = mtask;   // 0: Y, 1: Z, 2: E, 3: Zl
            if (sub == 0) {
                wrow[h][4][warp] = mb;
                wrow[h][5][warp] = mbeta;
            }
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) flags |= __shfl_xor_sync(0xffffffffu, flags, o);
    if (lane == 0 && flags) {
        if (flags & 1u) atomicOr(status, (unsigned long long)kStatusBadInput);
        if (flags & 2u) atomicOr(status, (unsigned long long)kStatusFp16Range);
    }
    __syncthreads();
    // centroids and boxes: the eight warps combined in a fixed order
    const int nvh0 = min(nv, 128), nvh1 = max(0, min(nv - 128, 128));
    for (int k = threadIdx.x; k < kPad; k += 256) {
        float sum[2] = {0.f, 0.f}, lo[2] = {INFINITY, INFINITY}, hi[2] = {-INFINITY, -INFINITY};
        for (int h = 0; h < halves; ++h)
#pragma unroll
            for (int w = 0; w < 8; ++w) {
                sum[h] += wsum[h][w][k];
                lo[h] = fminf(lo[h], wmin[h][w][k]);
                hi[h] = fmaxf(hi[h], wmax[h][w][k]);
            }
        const float c = (float)(((double)sum[0] + (double)sum[1]) / (double)max(nv, 1));
        cs[0][k] = c;
        if (k < d) {
            T.ctrT[(size_t)k * T.ntiles + t] = c;
            T.loT[(size_t)k * T.ntiles + t] = fminf(lo[0], lo[1]);
            T.hiT[(size_t)k * T.ntiles + t] = fmaxf(hi[0], hi[1]);
        }
        if (kHalves) {
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const float ch = (float)((double)sum[h] / (double)max(h ? nvh1 : nvh0, 1));
                cs[1 + h][k] = ch;
                if (k < d) {
                    const size_t e = (size_t)k * H.ntiles + 2 * t + h;
                    H.ctrT[e] = ch;
                    H.loT[e] = lo[h];
                    H.hiT[e] = hi[h];
                }
            }
        }
    }
    __syncthreads();
    // radius pass (the tile's rows again, from L2): FP32 sums of squared differences from the
    // centroids just written, bounded above as described at the top
    {
        float ct[kE], c0h[kE], c1h[kE];
#pragma unroll
        for (int q = 0; q < kE; ++q) {
            ct[q] = cs[0][k0 + q];
            c0h[q] = kHalves ? cs[1][k0 + q] : 0.f;
            c1h[q] = kHalves ? cs[2][k0 + q] : 0.f;
        }
        float mt = 0.f, mh0 = 0.f, mh1 = 0.f;
        for (int h = 0; h < halves; ++h) {
            const int hb = h * 128;
            if (hb >= nv) break;   // uniform
            for (int m0 = 0; m0 < kRows; m0 += kU) {
                float4 xv[kU][kV];
                int ii[kU];
#pragma unroll
                for (int u = 0; u < kU; ++u) {
                    ii[u] = hb + grp + (m0 + u) * kNG;
                    const bool ld = ii[u] < nv && kin;
                    const float4* rowp = ld ? reinterpret_cast<const float4*>(
                                                  src + (size_t)perm[r0 + ii[u]] * (size_t)d + k0)
                                            : nullptr;
#pragma unroll
                    for (int v = 0; v < kV; ++v)
                        xv[u][v] = (ld && k0 + 4 * v < d) ? __ldg(rowp + v) : make_float4(0.f, 0.f, 0.f, 0.f);
                }
#pragma unroll
                for (int u = 0; u < kU; ++u) {
                    float st_ = 0.f, sh = 0.f;
#pragma unroll
                    for (int q = 0; q < kE; ++q) {
                        const float4 f4 = xv[u][q / 4];
                        const float x = (q & 3) == 0 ? f4.x : (q & 3) == 1 ? f4.y : (q & 3) == 2 ? f4.z : f4.w;
                        const bool in = k0 + q < d;
                        const float df = in ? x - ct[q] : 0.f;
                        st_ = fmaf(df, df, st_);
                        if (kHalves) {
                            const float dh = in ? x - (h ? c1h[q] : c0h[q]) : 0.f;
                            sh = fmaf(dh, dh, sh);
                        }
                    }
#pragma unroll
                    for (int o = kL / 2; o > 0; o >>= 1) {
                        st_ += __shfl_xor_sync(0xffffffffu, st_, o);
                        if (kHalves) sh += __shfl_xor_sync(0xffffffffu, sh, o);
                    }
                    if (ii[u] < nv) {
                        mt = fmaxf(mt, st_);
                        if (kHalves) {
                            if (h) mh1 = fmaxf(mh1, sh);
                            else mh0 = fmaxf(mh0, sh);
                        }
                    }
                }
            }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            mt = fmaxf(mt, __shfl_xor_sync(0xffffffffu, mt, o));
            mh0 = fmaxf(mh0, __shfl_xor_sync(0xffffffffu, mh0, o));
            mh1 = fmaxf(mh1, __shfl_xor_sync(0xffffffffu, mh1, o));
        }
        if (lane == 0) {
            wrad[0][warp] = mt;
            wrad[1][warp] = mh0;
            wrad[2][warp] = mh1;
        }
    }
    __syncthreads();
    if (threadIdx.x < 3) {   // thread 0: the tile; threads 1, 2: the halves
        const int w = threadIdx.x;
        if (w == 0 || kHalves) {
            float m = 0.f;
#pragma unroll
            for (int q = 0; q < 8; ++q) m = fmaxf(m, wrad[w][q]);
            const int hv = w == 0 ? nv : (w == 1 ? nvh0 : nvh1);
            const float rb = hv > 0 ? __fsqrt_ru(__fmul_ru(__fadd_ru(m, slack32), up32)) : 0.f;
            float mx[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
            for (int q = 0; q < 6; ++q)
                for (int h = 0; h < halves; ++h) {
                    if (w > 0 && h != w - 1) continue;
#pragma unroll
                    for (int x = 0; x < 8; ++x) mx[q] = fmaxf(mx[q], wrow[h][q][x]);
                }
            TileOut& O = w == 0 ? T : H;
            const int e = w == 0 ? t : 2 * t + (w - 1);
            O.rad[e] = rb;
            O.maxY[e] = mx[0];
            O.maxZ[e] = mx[1];
            O.maxE[e] = mx[2];
            O.maxZl[e] = mx[3];
            O.maxB[e] = mx[4];
            O.beta[e] = mx[5];
            if (w > 0) {
                O.nvalid[e] = (uint32_t)hv;
                O.row0[e] = (uint32_t)(r0 + 128 * (w - 1));
            } else if (!tabled) {
                O.nvalid[e] = (uint32_t)max(nv, 0);
                O.row0[e] = (uint32_t)r0;
            }
        }
    }
}

// The fused operand pass for rows of at most 32 elements (kpad 16 or 32): one warp per tile, eight
// tiles per block, 4 elements per lane and 32 / kL rows per warp step; every combine is a shuffle, so
// the tile needs no shared memory and no block barrier (a 128-row tile of 8-element rows is 4 KB of
// input: a block per tile spent its time in barriers and serial combines).  The arithmetic is
// prep_row's, the statistics those of prep_tiles_kernel.
template <int kScreen, int kSplit, int kL, bool kHalves>
__global__ void __launch_bounds__(256, 3) prep_tiles_warp_kernel(const float* __restrict__ src, long long n, int d,
                                                              int tile, int ntiles, const uint32_t* __restrict__ perm,
                                                              const float* __restrict__ center,
                                                              const uint32_t* row0_in, const uint32_t* nvalid_in,
                                                              uint16_t* op, double* nrm2, float* nrm2f, float* zn,
                                                              float* en, float* yn, float* zl, TileOut T, TileOut H,
                                                              unsigned long long* status) {
    constexpr int kE = 4;
    constexpr int kRW = 32 / kL;               // rows per warp step
    constexpr int kSteps = 128 / kRW;          // steps per 128-row half
    constexpr int kRing = 16;                  // steps in flight
    static_assert(kL == 4 || kL == 8, "rows of 16 or 32 padded elements");
    extern __shared__ __align__(16) float4 pw_ring[];   // [8 warps][kRing][32 lanes]
    __shared__ uint32_t pw_perm[8][256];                 // the warp's tile rows' original ids
    const unsigned lane = threadIdx.x & 31;
    const int t = (int)blockIdx.x * 8 + (int)(threadIdx.x >> 5);
    if (t >= ntiles) return;   // whole warps; no block barrier in this kernel
    const bool tabled = row0_in != nullptr;
    const long long r0 = tabled ? (long long)row0_in[t] : (long long)t * tile;
    const int nv = tabled ? (int)nvalid_in[t] : (int)min((long long)tile, n - r0);
    const int halves = tile == 256 ? 2 : 1;
    const unsigned grp = lane / kL, sub = lane % kL;
    const int k0 = kE * (int)sub;
    const bool kin = k0 < d;
    float cf[kE];
    double cdv[kE];
#pragma unroll
    for (int q = 0; q < kE; ++q) {
        cf[q] = (k0 + q < d) ? center[k0 + q] : 0.f;
        cdv[q] = (double)cf[q];
    }
    const PrepBounds pb(d);
    unsigned flags = 0;
    // loads: the warp's rows stream through a per-lane ring of kRing 16-byte slots in shared memory
    // (cp.async, one commit group per step, kRing steps in flight), first for the statistics pass and
    // then again for the radius pass; the tile's permutation entries are staged first
    const int warp = (int)(threadIdx.x >> 5);
    float4* ring = pw_ring + (size_t)warp * kRing * 32 + lane;   // slot q at ring[32 q]
    uint32_t* wperm = pw_perm[warp];
    for (int k = (int)lane; k < nv; k += 32) wperm[k] = perm[r0 + k];
    __syncwarp();
    const int nh = nv > 128 && halves == 2 ? 2 : 1;
    const int pass_steps = nh * kSteps, total_steps = 2 * pass_steps;
    auto issue = [&](int q) {
        if (q < total_steps) {
            const int rem = q < pass_steps ? q : q - pass_steps;
            const int ii = (rem / kSteps) * 128 + (rem % kSteps) * kRW + (int)grp;
            if (ii < nv && kin) cp_async16(&ring[32 * (q % kRing)], src + (size_t)wperm[ii] * (size_t)d + k0);
        }
        cp_async_commit();
    };
#pragma unroll 1
    for (int q = 0; q < kRing; ++q) issue(q);
    int qc = 0;   // next step to consume
    // per half: the lane's centroid / box partials (combined over the warp's row groups below) and the
    // bound maxima (lanes 0-3 of a group: Y, Z, E, Zl; lane 0 also B and beta)
    float hs[2][kE], hl[2][kE], hh[2][kE], hm[2][6];
#pragma unroll
    for (int h = 0; h < 2; ++h) {
        float ps[kE], pl[kE], ph[kE];
#pragma unroll
        for (int q = 0; q < kE; ++q) { ps[q] = 0.f; pl[q] = INFINITY; ph[q] = -INFINITY; }
        float mtask = 0.f, mb = 0.f, mbeta = 0.f;
        if (h < nh) {   // uniform across the warp
#pragma unroll 1
            for (int s = 0; s < kSteps; ++s) {
                const int ii = h * 128 + s * kRW + (int)grp;
                cp_async_wait<kRing - 1>();
                const float4 xv = (ii < nv && kin) ? ring[32 * (qc % kRing)] : make_float4(0.f, 0.f, 0.f, 0.f);
                const float xa[kE] = {xv.x, xv.y, xv.z, xv.w};
                prep_row<kScreen, kSplit, kE, kL>(xa, cf, cdv, ii < nv, r0 + ii, k0, d, sub, lane, pb, op, nrm2,
                                                  nrm2f, zn, en, yn, zl, ps, pl, ph, mtask, mb, mbeta, flags);
                issue(qc + kRing);
                ++qc;
            }
        }
#pragma unroll
        for (int o = kL; o < 32; o <<= 1) {
#pragma unroll
            for (int q = 0; q < kE; ++q) {
                ps[q] += __shfl_xor_sync(0xffffffffu, ps[q], o);
                pl[q] = fminf(pl[q], __shfl_xor_sync(0xffffffffu, pl[q], o));
                ph[q] = fmaxf(ph[q], __shfl_xor_sync(0xffffffffu, ph[q], o));
            }
            mtask = fmaxf(mtask, __shfl_xor_sync(0xffffffffu, mtask, o));
            mb = fmaxf(mb, __shfl_xor_sync(0xffffffffu, mb, o));
            mbeta = fmaxf(mbeta, __shfl_xor_sync(0xffffffffu, mbeta, o));
        }
#pragma unroll
        for (int q = 0; q < kE; ++q) { hs[h][q] = ps[q]; hl[h][q] = pl[q]; hh[h][q] = ph[q]; }
        // bound maxima to every lane: Y, Z, E, Zl from lanes 0-3, B and beta from lane 0
#pragma unroll
        for (int b = 0; b < 4; ++b) hm[h][b] = __shfl_sync(0xffffffffu, mtask, b);
        hm[h][4] = __shfl_sync(0xffffffffu, mb, 0);
        hm[h][5] = __shfl_sync(0xffffffffu, mbeta, 0);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) flags |= __shfl_xor_sync(0xffffffffu, flags, o);
    if (lane == 0 && flags) {
        if (flags & 1u) atomicOr(status, (unsigned long long)kStatusBadInput);
        if (flags & 2u) atomicOr(status, (unsigned long long)kStatusFp16Range);
    }
    const int nvh0 = min(nv, 128), nvh1 = max(0, min(nv - 128, 128));
    float ct[kE], c0h[kE], c1h[kE];
#pragma unroll
    for (int q = 0; q < kE; ++q) {
        const int k = k0 + q;
        ct[q] = (float)(((double)hs[0][q] + (double)hs[1][q]) / (double)max(nv, 1));
        c0h[q] = (float)((double)hs[0][q] / (double)max(nvh0, 1));
        c1h[q] = (float)((double)hs[1][q] / (double)max(nvh1, 1));
        if (grp == 0 && k < d) {
            T.ctrT[(size_t)k * T.ntiles + t] = ct[q];
            T.loT[(size_t)k * T.ntiles + t] = fminf(hl[0][q], hl[1][q]);
            T.hiT[(size_t)k * T.ntiles + t] = fmaxf(hh[0][q], hh[1][q]);
            if (kHalves) {
                const size_t e0 = (size_t)k * H.ntiles + 2 * t;
                H.ctrT[e0] = c0h[q];
                H.loT[e0] = hl[0][q];
                H.hiT[e0] = hh[0][q];
                H.ctrT[e0 + 1] = c1h[q];
                H.loT[e0 + 1] = hl[1][q];
                H.hiT[e0 + 1] = hh[1][q];
            }
        }
    }
    // radius pass (the tile's rows again, from L2 through the ring), bounded as in prep_tiles_kernel
    float mt = 0.f, mh0 = 0.f, mh1 = 0.f;
    for (int h = 0; h < nh; ++h) {
#pragma unroll 1
        for (int s = 0; s < kSteps; ++s) {
            const int ii = h * 128 + s * kRW + (int)grp;
            cp_async_wait<kRing - 1>();
            const float4 xv = (ii < nv && kin) ? ring[32 * (qc % kRing)] : make_float4(0.f, 0.f, 0.f, 0.f);
            {
                const float xa[kE] = {xv.x, xv.y, xv.z, xv.w};
                float st_ = 0.f, sh = 0.f;
#pragma unroll
                for (int q = 0; q < kE; ++q) {
                    const bool in = k0 + q < d;
                    const float df = in ? xa[q] - ct[q] : 0.f;
                    st_ = fmaf(df, df, st_);
                    if (kHalves) {
                        const float dh = in ? xa[q] - (h ? c1h[q] : c0h[q]) : 0.f;
                        sh = fmaf(dh, dh, sh);
                    }
                }
#pragma unroll
                for (int o = kL / 2; o > 0; o >>= 1) {
                    st_ += __shfl_xor_sync(0xffffffffu, st_, o);
                    if (kHalves) sh += __shfl_xor_sync(0xffffffffu, sh, o);
                }
                if (ii < nv) {
                    mt = fmaxf(mt, st_);
                    if (kHalves) {
                        if (h) mh1 = fmaxf(mh1, sh);
                        else mh0 = fmaxf(mh0, sh);
                    }
                }
            }
            issue(qc + kRing);
            ++qc;
        }
    }
    cp_async_wait<0>();   // the ring's trailing (empty) groups
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        mt = fmaxf(mt, __shfl_xor_sync(0xffffffffu, mt, o));
        mh0 = fmaxf(mh0, __shfl_xor_sync(0xffffffffu, mh0, o));
        mh1 = fmaxf(mh1, __shfl_xor_sync(0xffffffffu, mh1, o));
    }
    if (lane < 3 && (lane == 0 || kHalves)) {   // lane 0: the tile; lanes 1, 2: the halves
        const int w = (int)lane;
        const float m = w == 0 ? mt : (w == 1 ? mh0 : mh1);
        const int hv = w == 0 ? nv : (w == 1 ? nvh0 : nvh1);
        TileOut& O = w == 0 ? T : H;
        const int e = w == 0 ? t : 2 * t + (w - 1);
        O.rad[e] = hv > 0 ? __fsqrt_ru(__fmul_ru(__fadd_ru(m, pb.slack32), pb.up32)) : 0.f;
        float mx[6];
#pragma unroll
        for (int q = 0; q < 6; ++q)
            mx[q] = w == 0 ? fmaxf(hm[0][q], hm[1][q]) : (w == 1 ? hm[0][q] : hm[1][q]);
        O.maxY[e] = mx[0];
        O.maxZ[e] = mx[1];
        O.maxE[e] = mx[2];
        O.maxZl[e] = mx[3];
        O.maxB[e] = mx[4];
        O.beta[e] = mx[5];
        if (w > 0) {
            O.nvalid[e] = (uint32_t)hv;
            O.row0[e] = (uint32_t)(r0 + 128 * (w - 1));
        } else if (!tabled) {
            O.nvalid[e] = (uint32_t)max(nv, 0);
            O.row0[e] = (uint32_t)r0;
        }
    }
}

// Candidate test: thread = one S tile J, 16 R tiles per block (from shared memory).
// Keeps (I, J) unless a rigorous lower bound on every pair distance exceeds sqrt(Tp).
template <int kCandI>
__global__ void __launch_bounds__(256) cand_test(const float* rctrT, const float* rloT, const float* rhiT,
                                                 const float* rrad, int ntR, const float* sctrT,
                                                 const float* sloT, const float* shiT, const float* srad, int ntS,
                                                 int d, int tileR, int tileS, double Tp, int self_join,
                                                 uint32_t* bitmap, int words) {
    extern __shared__ float sm[];   // [3][kCandI][d]
    float* sc = sm;
    float* slo = sm + kCandI * d;
    float* shi = sm + 2 * kCandI * d;
    const int I0 = blockIdx.y * kCandI;
    const int nI = min(kCandI, ntR - I0);
    for (int e = threadIdx.x; e < kCandI * d; e += blockDim.x) {
        const int ii = e / d, k = e % d;
        const bool ok = ii < nI;
        sc[e] = ok ? rctrT[(size_t)k * ntR + I0 + ii] : 0.f;
        slo[e] = ok ? rloT[(size_t)k * ntR + I0 + ii] : 0.f;
        shi[e] = ok ? rhiT[(size_t)k * ntR + I0 + ii] : 0.f;
    }
    __syncthreads();
    const int J = blockIdx.x * blockDim.x + threadIdx.x;
    const bool jok = J < ntS;
    float ball[kCandI], box[kCandI];
#pragma unroll
    for (int ii = 0; ii < kCandI; ++ii) ball[ii] = box[ii] = 0.f;
    if (jok) {
        for (int k = 0; k < d; ++k) {
            const float cj = sctrT[(size_t)k * ntS + J];
            const float lj = sloT[(size_t)k * ntS + J];
            const float hj = shiT[(size_t)k * ntS + J];
#pragma unroll
            for (int ii = 0; ii < kCandI; ++ii) {
                const float dc = sc[ii * d + k] - cj;
                ball[ii] = fmaf(dc, dc, ball[ii]);
                const float gap = fmaxf(fmaxf(lj - shi[ii * d + k], slo[ii * d + k] - hj), 0.f);
                box[ii] = fmaf(gap, gap, box[ii]);
            }
        }
    }
    // FP32 sums of d non-negative terms: computed >= (1 - (d+4) 2^-23) * true  => true >= computed * f
    const float f = 1.f - (float)(d + 8) * 0x1p-23f;
    const float rtp = (float)(sqrt(Tp) * (1.0 + 0x1p-20));
    const float tpf = (float)(Tp * (1.0 + 0x1p-20));
    const float rj = jok ? srad[J] : 0.f;
    const unsigned lane = threadIdx.x & 31;
    for (int ii = 0; ii < kCandI; ++ii) {
        const int I = I0 + ii;
        bool keep = jok && ii < nI;
        if (keep && self_join) {
            // some column index of J must exceed some row index of I (sorted positions)
            const long long maxcol = (long long)(J + 1) * tileS - 1;
            keep = maxcol > (long long)I * tileR;
        }
        if (keep) {
            const float lb_box = box[ii] * f;
            const float lb_ball = sqrtf(ball[ii] * f) * (1.f - 0x1p-20f) - rrad[I] - rj;
            if (lb_box > tpf || lb_ball > rtp) keep = false;
        }
        const unsigned bits = __ballot_sync(0xffffffffu, keep);
        if (lane == 0 && ii < nI && (J >> 5) < words) bitmap[(size_t)I * words + (J >> 5)] = bits;
    }
}

// Batched candidate test: one block = up to kCandI R tiles of one join against all S tiles of
// the same join (tiles of different joins never pair).  Same rigorous bounds as cand_test.
template <int kCandI>
__global__ void __launch_bounds__(256) cand_test_batched(const CandBlock* blocks, const CandClassView* views,
                                                         const double* Tp_blk, uint32_t* bitmap, int words) {
    extern __shared__ float sm[];   // [3][kCandI][d]
    const CandBlock cb = blocks[blockIdx.x];
    const CandClassView cv = views[cb.cls];
    const int d = cv.d;
    float* sc = sm;
    float* slo = sm + kCandI * d;
    float* shi = sm + 2 * kCandI * d;
    const int iloc0 = (int)cb.i0 - cv.rbase;   // class-local R tile of the block's first tile
    for (int e = threadIdx.x; e < kCandI * d; e += blockDim.x) {
        const int ii = e / d, k = e % d;
        const bool ok = ii < (int)cb.ni;
        sc[e] = ok ? cv.rctrT[(size_t)k * cv.ntR + iloc0 + ii] : 0.f;
        slo[e] = ok ? cv.rloT[(size_t)k * cv.ntR + iloc0 + ii] : 0.f;
        shi[e] = ok ? cv.rhiT[(size_t)k * cv.ntR + iloc0 + ii] : 0.f;
    }
    __syncthreads();
    const double Tp = Tp_blk[blockIdx.x];
    const float f = 1.f - (float)(d + 8) * 0x1p-23f;
    const float rtp = (float)(sqrt(Tp) * (1.0 + 0x1p-20));
    const float tpf = (float)(Tp * (1.0 + 0x1p-20));
    const unsigned lane = threadIdx.x & 31;
    for (int j0 = 0; j0 < (int)cb.nj; j0 += blockDim.x) {
        const int jl = j0 + threadIdx.x;          // S tile index inside the join
        const bool jok = jl < (int)cb.nj;
        const int js = (int)cb.j0 - cv.sbase + jl;   // class-local S tile
        float ball[kCandI], box[kCandI];
#pragma unroll
        for (int ii = 0; ii < kCandI; ++ii) ball[ii] = box[ii] = 0.f;
        if (jok) {
            for (int k = 0; k < d; ++k) {
                const float cj = cv.sctrT[(size_t)k * cv.ntS + js];
                const float lj = cv.sloT[(size_t)k * cv.ntS + js];
                const float hj = cv.shiT[(size_t)k * cv.ntS + js];
#pragma unroll
                for (int ii = 0; ii < kCandI; ++ii) {
                    const float dc = sc[ii * d + k] - cj;
                    ball[ii] = fmaf(dc, dc, ball[ii]);
                    const float gap = fmaxf(fmaxf(lj - shi[ii * d + k], slo[ii * d + k] - hj), 0.f);
                    box[ii] = fmaf(gap, gap, box[ii]);
                }
            }
        }
        const float rj = jok ? cv.srad[js] : 0.f;
        for (int ii = 0; ii < kCandI; ++ii) {
            bool keep = jok && ii < (int)cb.ni;
            if (keep) {
                const float lb_box = box[ii] * f;
                const float lb_ball = sqrtf(ball[ii] * f) * (1.f - 0x1p-20f) - cv.rrad[iloc0 + ii] - rj;
                if (lb_box > tpf || lb_ball > rtp) keep = false;
            }
            const unsigned bits = __ballot_sync(0xffffffffu, keep);
            if (lane == 0 && ii < (int)cb.ni && (jl >> 5) < words)
                bitmap[(size_t)(cb.i0 + ii) * words + (jl >> 5)] = bits;
        }
    }
}

__global__ void cand_count(const uint32_t* bitmap, int words, int ntR, uint32_t* cnt) {
    const int I = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const unsigned lane = threadIdx.x & 31;
    if (I >= ntR) return;
    unsigned c = 0;
    for (int w = lane; w < words; w += 32) c += __popc(bitmap[(size_t)I * words + w]);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
    if (lane == 0) cnt[I] = c;
}

__global__ void cand_fill(const uint32_t* bitmap, int words, int ntR, const uint32_t* off, uint32_t* jlist,
                          const uint32_t* rtile_sbase) {
    const int I = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const unsigned lane = threadIdx.x & 31;
    if (I >= ntR) return;
    uint32_t pos = off[I];
    const uint32_t sb = rtile_sbase ? rtile_sbase[I] : 0u;   // batched: global id of the join's first S tile
    for (int w0 = 0; w0 < words; w0 += 32) {
        const int w = w0 + lane;
        const unsigned bits = w < words ? bitmap[(size_t)I * words + w] : 0u;
        unsigned tot;
        const unsigned pre = warp_excl_scan(__popc(bits), tot);
        unsigned b = bits, p = pos + pre;
        while (b) {
            const int bit = __ffs(b) - 1;
            b &= b - 1;
            jlist[p++] = sb + (uint32_t)(w * 32 + bit);
        }
        pos += tot;
    }
}

__global__ void chunk_counts(const uint32_t* cnt, int ntR, int ch, uint32_t* nch) {
    const int I = blockIdx.x * blockDim.x + threadIdx.x;
    if (I < ntR) nch[I] = (cnt[I] + ch - 1) / ch;
}

// Emit one (w, I) sort key per chunk; unused capacity gets the max key.
__global__ void chunk_keys(const uint32_t* nch, const uint32_t* cbase, int ntR, size_t cap, uint64_t* keys,
                           uint32_t* vals) {
    const int I = blockIdx.x * blockDim.x + threadIdx.x;
    if (I >= ntR) return;
    const uint32_t b = cbase[I], c = nch[I];
    for (uint32_t w = 0; w < c; ++w) {
        if (b + w < cap) {
            keys[b + w] = ((uint64_t)w << 32) | (uint32_t)I;
            vals[b + w] = b + w;
        }
    }
}

__global__ void fill_keys_max(uint64_t* keys, uint32_t* vals, size_t from, size_t cap, const uint32_t* total) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x + from;
    if (i < cap && i >= *total) {
        keys[i] = ~0ull;
        vals[i] = 0xFFFFFFFFu;
    }
}

__global__ void chunk_emit(const uint64_t* keys, size_t cap, const uint32_t* total, const uint32_t* cnt,
                           const uint32_t* off, int ch, uint4* chunks) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= cap) return;
    if (i >= *total) return;
    const uint64_t k = keys[i];
    const uint32_t I = (uint32_t)(k & 0xFFFFFFFFu), w = (uint32_t)(k >> 32);
    const uint32_t b = off[I] + w * (uint32_t)ch;
    const uint32_t e = min(b + (uint32_t)ch, off[I] + cnt[I]);
    chunks[i] = make_uint4(I, b, e, 0);
}

// Half-tile masks for the one-SM tensor-core screen.  A candidate (R tile I, S tile J) of 128 x 256
// rows is issued as two 128-column half-items; this tests each 128-row half of S tile J against R
// tile I with cand_test's rigorous ball and box bounds (on the halves' own statistics) and stores the
// live halves in bits 30-31 of the jlist entry.  The screen then issues and tests only live halves,
// packing them densely into its MMA and epilogue pipeline; an entry whose halves are both dead is
// skipped.  Warps stride over the scheduling chunks (at most chunk_items candidates of one R tile),
// the chunk's R tile statistics in the warp's shared memory, and take its candidates one at a time
// with the lanes over the dimensions; the halves' statistics are read row-major, so each load of
// the warp is one contiguous run of a candidate's row.
__global__ void __launch_bounds__(256) half_mask_kernel(const uint4* chunks, const uint32_t* nchunks, uint32_t* jlist,
                                                        const uint4* rtiles, const JoinParams* jps,
                                                        const HalfView* views, int self_join, int dmax) {
    extern __shared__ float hm_sm[];   // [8 warps][3][dmax]: R tile centroid, low, high
    const unsigned warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    float* rs = hm_sm + (size_t)warp * 3 * dmax;
    const unsigned nch = *nchunks;
    for (unsigned ci = blockIdx.x * 8 + warp; ci < nch; ci += gridDim.x * 8) {   // warp-uniform
        const uint4 ch = chunks[ci];
        const int I = (int)ch.x;
        const uint4 rt = rtiles[I];
        const HalfView v = views[rt.w];
        const int d = v.d;
        const int il = I - v.rbase;   // class-local R tile
        __syncwarp();                  // the previous chunk's reads of rs are done
        for (int k = lane; k < d; k += 32) {
            rs[k] = v.rctrT[(size_t)k * v.ntR + il];
            rs[d + k] = v.rloT[(size_t)k * v.ntR + il];
            rs[2 * d + k] = v.rhiT[(size_t)k * v.ntR + il];
        }
        __syncwarp();
        const double Tp = jps[rt.z].Tp;
        const float f = 1.f - (float)(d + 8) * 0x1p-23f;
        const float rtp = (float)(sqrt(Tp) * (1.0 + 0x1p-20));
        const float tpf = (float)(Tp * (1.0 + 0x1p-20));
        const float ri = v.rrad[il];
        // one candidate at a time, the warp's lanes over its dimensions (coalesced reads of the
        // halves' row-major statistics whatever tiles the candidates are), sums by a shuffle tree
        for (uint32_t e = ch.y; e < ch.z; ++e) {   // warp-uniform
            const uint32_t J = jlist[e] & 0x3FFFFFFFu;
            const int h0 = 2 * ((int)J - v.sbase);   // class-local half tiles h0, h0 + 1
            bool live[2];
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                live[h] = h0 + h < v.ntH && v.hnv[h0 + h] != 0;
                // self-joins: some sorted column of the half must exceed some sorted row of the tile
                if (self_join && (long long)(h0 + h) * 128 + 127 <= (long long)il * 128) live[h] = false;
            }
            const int g0 = live[0] ? h0 : h0 + 1, g1 = live[1] ? h0 + 1 : h0;   // in-range rows for both
            float ball[2] = {0.f, 0.f}, box[2] = {0.f, 0.f};
            if (live[0] || live[1]) {
                const float *c0 = v.hctrR + (size_t)g0 * d, *c1 = v.hctrR + (size_t)g1 * d;
                const float *l0 = v.hloR + (size_t)g0 * d, *l1 = v.hloR + (size_t)g1 * d;
                const float *u0 = v.hhiR + (size_t)g0 * d, *u1 = v.hhiR + (size_t)g1 * d;
                for (int k = lane; k < d; k += 32) {
                    const float c = rs[k], lo = rs[d + k], hi = rs[2 * d + k];
                    const float dc0 = c - c0[k], dc1 = c - c1[k];
                    const float gp0 = fmaxf(fmaxf(l0[k] - hi, lo - u0[k]), 0.f);
                    const float gp1 = fmaxf(fmaxf(l1[k] - hi, lo - u1[k]), 0.f);
                    ball[0] = fmaf(dc0, dc0, ball[0]);
                    ball[1] = fmaf(dc1, dc1, ball[1]);
                    box[0] = fmaf(gp0, gp0, box[0]);
                    box[1] = fmaf(gp1, gp1, box[1]);
                }
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) {
                    ball[0] += __shfl_xor_sync(0xffffffffu, ball[0], o);
                    ball[1] += __shfl_xor_sync(0xffffffffu, ball[1], o);
                    box[0] += __shfl_xor_sync(0xffffffffu, box[0], o);
                    box[1] += __shfl_xor_sync(0xffffffffu, box[1], o);
                }
            }
            // each partial sum is a sum of non-negative FP32 terms, one more rounding per shuffle
            // level: the deflation by f = 1 - (d + 8) 2^-23 covers d + 5 roundings
            unsigned mask = 0;
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                if (!live[h]) continue;
                const float lb_box = box[h] * f;
                const float lb_ball = sqrtf(ball[h] * f) * (1.f - 0x1p-20f) - ri - v.hrad[h0 + h];
                if (!(lb_box > tpf || lb_ball > rtp)) mask |= 1u << h;
            }
            if (lane == 0) jlist[e] = J | (mask << 30);
        }
    }
}

// [d][nt] -> [nt][d] for the three per-dimension statistics of a tile set.
__global__ void stats_rowmajor_kernel(const float* ctrT, const float* loT, const float* hiT, int nt, int d, float* ctrR,
                                      float* loR, float* hiR) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;   // row-major index t * d + k
    if (i >= (size_t)nt * d) return;
    const size_t t = i / (size_t)d, k = i - t * (size_t)d;
    ctrR[i] = ctrT[k * nt + t];
    loR[i] = loT[k * nt + t];
    hiR[i] = hiT[k * nt + t];
}

}  // namespace

// ------------------------------------------------------------------ host entry points

bool compute_frame(const void* const* srcs, const long long* ns, int nsrc, int d, int dtype, int frame_mode,
                   FrameParams* fp, float* center, cudaStream_t st) {
    // The per-dimension statistics choose the Morton frame and the centre c; any centre and any frame
    // leave the pairs unchanged (the certificate is computed from the operands actually formed, and
    // cell coordinates outside the measured range are clamped), so they come from an evenly strided
    // sample of at most kStatSampleRows rows per side.
    constexpr long long kStatSampleRows = 1ll << 16;
    long long ntot = 0, nstat = 0;
    std::vector<long long> rstride(nsrc), nsampled(nsrc);
    for (int s = 0; s < nsrc; ++s) {
        ntot += ns[s];
        rstride[s] = std::max(1ll, ns[s] / kStatSampleRows);
        nsampled[s] = (ns[s] + rstride[s] - 1) / rstride[s];   // (nsampled - 1) * rstride < ns
        nstat += nsampled[s];
    }
    const int parts = nsrc * kStatBlocks;
    DBuf<float> pmin((size_t)parts * d, st), pmax((size_t)parts * d, st);
    DBuf<double> psum((size_t)parts * d, st), psq((size_t)parts * d, st);
    DBuf<float> ws((size_t)3 * d, st);
    for (int s = 0; s < nsrc; ++s) {
        const int nb = kStatBlocks;
        launch(dim_stats_partial, nb, 256, 0, st, srcs[s], dtype, nsampled[s], rstride[s], d, pmin.p, pmax.p, psum.p,
               psq.p, s * kStatBlocks);
    }
    launch(dim_reduce, (unsigned)d, 256, 0, st, pmin.p, pmax.p, psum.p, psq.p, parts, nstat, d, ws.p,
           ws.p + d, ws.p + 2 * d, center);
    const bool pca = frame_mode != kFrameAxes && d >= 9 && d <= kPcaMaxD && ntot > 0 &&
                     (frame_mode == kFramePca || ntot >= kPcaMinRows);
    if (pca) {   // principal-component cells
        const long long stride = std::max(1ll, ntot / kPcaSamples);
        const long long nsamp = (ntot + stride - 1) / stride;   // (nsamp - 1) * stride < ntot
        std::vector<long long> offs(nsrc + 1, 0);
        for (int s = 0; s < nsrc; ++s) offs[s + 1] = offs[s] + ns[s];
        DBuf<const void*> dsrc((size_t)nsrc, st);
        DBuf<long long> doff((size_t)nsrc + 1, st);
        upload(dsrc.p, srcs, nsrc * sizeof(void*), st);
        upload(doff.p, offs.data(), (nsrc + 1) * sizeof(long long), st);
        DBuf<float> part((size_t)kCovBlocks * d * d, st);   // >= kCovBlocks * 16 floats (d >= 9)
        DBuf<float> cov((size_t)d * d, st);
        launch(cov_partial, kCovBlocks, 256, 0, st, (const void* const*)dsrc.p, (const long long*)doff.p, nsrc,
               stride, nsamp, d, dtype, (const float*)center, part.p);
        launch(cov_reduce, (unsigned)((d * d + 255) / 256), 256, 0, st, (const float*)part.p, kCovBlocks, d * d,
               cov.p);
        const size_t smem = (size_t)(d * d + 16 * d) * sizeof(float);
        if (smem > 48 * 1024)
            TJ_CUDA(cudaFuncSetAttribute(pca_frame, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        launch(pca_frame, 1, 256, smem, st, (const float*)cov.p, d, fp);
        launch(proj_range_partial, kCovBlocks, 256, 0, st, (const void* const*)dsrc.p, (const long long*)doff.p,
               nsrc, stride, nsamp, d, dtype, (const float*)center, (const FrameParams*)fp, part.p);
        launch(pca_range_finish, 1, 32, 0, st, (const float*)part.p, kCovBlocks, fp);
    } else {
        launch(frame_pick, 1, 32, 0, st, d, ws.p, ws.p + d, ws.p + 2 * d, fp);
    }
    TJ_CUDA(cudaGetLastError());
    return pca;
}

namespace {

// Device arrays of a tile set (tables uploaded when the host built them).
void alloc_tiles(TileSet& ts, int tile, int d, int ntiles, cudaStream_t st) {
    ts.tile = tile;
    ts.d = d;
    ts.ntiles = ntiles;
    const size_t nt = (size_t)std::max(ntiles, 1);
    ts.ctrT = DBuf<float>(nt * d, st);
    ts.loT = DBuf<float>(nt * d, st);
    ts.hiT = DBuf<float>(nt * d, st);
    ts.rad = DBuf<float>(nt, st);
    ts.maxZ = DBuf<float>(nt, st);
    ts.maxE = DBuf<float>(nt, st);
    ts.maxY = DBuf<float>(nt, st);
    ts.maxB = DBuf<float>(nt, st);
    ts.beta = DBuf<float>(nt, st);
    ts.maxZl = DBuf<float>(nt, st);
    ts.nvalid = DBuf<uint32_t>(nt, st);
    ts.row0 = DBuf<uint32_t>(nt, st);
    if (ntiles > 0 && !ts.h_row0.empty()) {
        upload(ts.row0.p, ts.h_row0.data(), nt * 4, st);
        upload(ts.nvalid.p, ts.h_nvalid.data(), nt * 4, st);
    }
}

TileOut tile_out(TileSet& ts) {
    return TileOut{ts.ctrT.p, ts.loT.p, ts.hiT.p, ts.rad.p, ts.maxZ.p, ts.maxE.p, ts.maxY.p, ts.maxB.p,
                   ts.beta.p, ts.maxZl.p, ts.nvalid.p, ts.row0.p, ts.ntiles};
}

bool fused_prep_ok(const Side& s) {
    const bool f16 = s.screen == kScreenBF16 || s.screen == kScreenFP16 || s.screen == kScreenBF16X3 ||
                     s.screen == kScreenFP16X3;
    return f16 && s.dtype == kF32 && s.d % 4 == 0 && s.kpad <= 128 && ((uintptr_t)s.src & 15u) == 0;
}

// The fused pass over one tiling of the side (operands, norms, bounds and tile statistics).
void prep_tiles(Side& s, const float* center, int tile, TileSet& ts, TileSet* halves, cudaStream_t st,
                unsigned long long* status) {
    const bool tabled = !ts.h_row0.empty();
    const int ntiles = tabled ? (int)ts.h_row0.size() : (int)((s.n + tile - 1) / tile);
    alloc_tiles(ts, tile, s.d, ntiles, st);
    TileOut H{};
    if (halves) {
        halves->h_row0.clear();
        halves->h_nvalid.clear();
        alloc_tiles(*halves, 128, s.d, 2 * ntiles, st);
        H = tile_out(*halves);
        halves->built = true;
    }
    ts.built = true;
    // rows past the last tile (the operand padding up to rows_pad) are zero
    const long long n = s.n, rp = s.rows_pad;
    if (rp > n) {
        const size_t opw = (size_t)s.kpad * (s.split ? 2 : 1);
        TJ_CUDA(cudaMemsetAsync(s.op.p + (size_t)n * opw, 0, (size_t)(rp - n) * opw * sizeof(uint16_t), st));
        TJ_CUDA(cudaMemsetAsync(s.nrm2.p + n, 0, (size_t)(rp - n) * sizeof(double), st));
        float* fl[5] = {s.nrm2f.p, s.zn.p, s.en.p, s.yn.p, s.zl.p};
        for (float* f : fl) TJ_CUDA(cudaMemsetAsync(f + n, 0, (size_t)(rp - n) * sizeof(float), st));
    }
    if (ntiles == 0) return;
    const uint32_t* r0 = tabled ? (const uint32_t*)ts.row0.p : nullptr;
    const uint32_t* nvv = tabled ? (const uint32_t*)ts.nvalid.p : nullptr;
    const TileOut T = tile_out(ts);
#define TJ_PT(SCR, SPLIT, E, L, HV)                                                                                 \
    launch(prep_tiles_kernel<SCR, SPLIT, E, L, HV>, (unsigned)ntiles, 256, 0, st, (const float*)s.src, n, s.d, tile, \
           (const uint32_t*)s.perm.p, center, r0, nvv, s.op.p, s.nrm2.p, s.nrm2f.p, s.zn.p, s.en.p, s.yn.p,      \
           s.zl.p, T, H, status)
#define TJ_PTW(SCR, SPLIT, L, HV)                                                                                 \
    do {                                                                                                          \
        const int ring_bytes = 8 * 16 * 32 * 16;                                                                  \
        TJ_CUDA(cudaFuncSetAttribute(prep_tiles_warp_kernel<SCR, SPLIT, L, HV>,                                   \
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, ring_bytes));                   \
        TJ_CUDA(cudaFuncSetAttribute(prep_tiles_warp_kernel<SCR, SPLIT, L, HV>,                                   \
                                     cudaFuncAttributePreferredSharedMemoryCarveout, 100));                       \
        launch(prep_tiles_warp_kernel<SCR, SPLIT, L, HV>, (unsigned)((ntiles + 7) / 8), 256, ring_bytes, st,      \
               (const float*)s.src, n, s.d, tile, ntiles, (const uint32_t*)s.perm.p, center, r0, nvv, s.op.p,     \
               s.nrm2.p, s.nrm2f.p, s.zn.p, s.en.p, s.yn.p, s.zl.p, T, H, status);                               \
    } while (0)
#define TJ_PT_L(SCR, SPLIT, HV)                                  \
    do {                                                         \
        if (s.kpad == 16) TJ_PTW(SCR, SPLIT, 4, HV);             \
        else if (s.kpad == 32) TJ_PTW(SCR, SPLIT, 8, HV);        \
        else if (s.kpad == 64) TJ_PT(SCR, SPLIT, 8, 8, HV);      \
        else TJ_PT(SCR, SPLIT, 8, 16, HV);                       \
    } while (0)
#define TJ_PT_H(SCR, SPLIT)                                      \
    do {                                                         \
        if (halves) TJ_PT_L(SCR, SPLIT, true);                   \
        else TJ_PT_L(SCR, SPLIT, false);                         \
    } while (0)
    switch (s.screen) {
        case kScreenBF16: TJ_PT_H(kScreenBF16, 0); break;
        case kScreenFP16: TJ_PT_H(kScreenFP16, 0); break;
        case kScreenBF16X3: TJ_PT_H(kScreenBF16X3, 1); break;
        default: TJ_PT_H(kScreenFP16X3, 1); break;
    }
#undef TJ_PT_H
#undef TJ_PT_L
#undef TJ_PTW
#undef TJ_PT
}

}  // namespace

void prepare_side(Side& s, const FrameParams* fpd, bool pca_frame, const float* center, cudaStream_t st,
                  unsigned long long* status, TileSet* ts, int tile, TileSet* halves) {
    const long long n = s.n;
    const bool i8 = s.screen == kScreenInt8Limb;
    s.split = (s.screen == kScreenBF16X3 || s.screen == kScreenFP16X3) ? 1 : 0;
    // 16-bit operands: rows of 16 or 32 elements for small d (32- / 64-byte swizzle), else a
    // multiple of 64 (128-byte swizzle); int8 limbs: a multiple of 128
    s.kpad = i8 ? ((s.d + 127) / 128) * 128
                : s.d <= 16 ? 16 : s.d <= 32 ? 32 : ((s.d + kBK - 1) / kBK) * kBK;
    s.rows_pad = ((std::max<long long>(n, 1) + kTileS - 1) / kTileS) * kTileS;
    s.perm = DBuf<uint32_t>((size_t)std::max<long long>(n, 1), st);
    s.keys = DBuf<uint64_t>((size_t)std::max<long long>(n, 1), st);
    if (n > 0) {
        DBuf<uint64_t> ktmp((size_t)n, st);
        DBuf<uint32_t> vtmp((size_t)n, st);
        DBuf<uint32_t> ws(radix_workspace_elems((size_t)n), st);
        if (pca_frame)
            launch(morton_keys_pca, (unsigned)((n + 255) / 256), 256, 0, st, s.src, s.dtype, n, s.d, fpd, s.keys.p,
                   s.perm.p, s.d_rowoff, s.njc, center);
        else
            launch(morton_keys, (unsigned)((n + 255) / 256), 256, 0, st, s.src, s.dtype, n, s.d, fpd, s.keys.p,
                   s.perm.p, s.d_rowoff, s.njc);
        int jbits = 0;
        while ((1 << jbits) < s.njc) ++jbits;
        bool in_tmp = false;
        radix_sort(s.keys.p, s.perm.p, ktmp.p, vtmp.p, (size_t)n, 32 + jbits, ws.p, st, status, &in_tmp);
        if (in_tmp) {   // odd number of passes: the sorted arrays are the temporaries
            std::swap(s.keys, ktmp);
            std::swap(s.perm, vtmp);
        }
        // joins on int14 rows (one join, 128-row tiles): rows inside each tile by norm (the sorted
        // keys are not read again on this path)
        if (i8 && ts && tile == 128 && s.njc <= 1)
            launch(order_tile_rows_by_norm, (unsigned)((n + 127) / 128), 128, 0, st, s.src, s.dtype, n, s.d,
                   s.perm.p);
    }
    s.emit = s.perm.p;
    const size_t rp = (size_t)s.rows_pad;
    const bool f16 = !i8 && s.screen != kScreenPlain;
    if (f16) s.op = DBuf<uint16_t>(rp * (size_t)s.kpad * (s.split ? 2 : 1), st);
    if (i8) {
        s.op8 = DBuf<int8_t>(rp * 2 * s.kpad, st);
        s.inorm = DBuf<long long>(rp, st);
    }
    if (s.screen == kScreenPlain) s.xs = DBuf<float>(rp * s.d, st);
    s.nrm2 = DBuf<double>(rp, st);
    s.nrm2f = DBuf<float>(rp, st);
    s.zn = DBuf<float>(rp, st);
    s.en = DBuf<float>(rp, st);
    s.yn = DBuf<float>(rp, st);
    s.zl = DBuf<float>(rp, st);
    if (ts && fused_prep_ok(s) && (tile == 128 || tile == 256) && (!halves || tile == 256)) {
        prep_tiles(s, center, tile, *ts, halves, st, status);
        return;
    }
    // lanes per row: 4 for rows of <= 16 elements, 8 for <= 32, else a warp
#define TJ_PREP_L(SCR, SPLIT, L)                                                                                 \
    launch(prep_rows<SCR, SPLIT, L>, (unsigned)((rp * L + 255) / 256), 256, 0, st, s.src, s.dtype, n, s.d, s.kpad, \
           s.rows_pad, s.perm.p, center, s.op.p, s.op8.p, s.xs.p, s.nrm2.p, s.nrm2f.p, s.zn.p, s.en.p, s.yn.p,      \
           s.zl.p, s.inorm.p, status)
#define TJ_PREP(SCR, SPLIT)                                    \
    do {                                                       \
        if (s.kpad <= 16) TJ_PREP_L(SCR, SPLIT, 4);            \
        else if (s.kpad <= 32) TJ_PREP_L(SCR, SPLIT, 8);       \
        else TJ_PREP_L(SCR, SPLIT, 32);                        \
    } while (0)
    switch (s.screen) {
        case kScreenPlain: TJ_PREP(kScreenPlain, 0); break;
        case kScreenBF16: TJ_PREP(kScreenBF16, 0); break;
        case kScreenFP16: TJ_PREP(kScreenFP16, 0); break;
        case kScreenBF16X3: TJ_PREP(kScreenBF16X3, 1); break;
        case kScreenFP16X3: TJ_PREP(kScreenFP16X3, 1); break;
        default: TJ_PREP(kScreenInt8Limb, 0); break;
    }
#undef TJ_PREP
#undef TJ_PREP_L
}

void tile_stats(const Side& s, int tile, TileSet& ts, cudaStream_t st) {
    if (ts.built) return;   // made by the fused operand pass
    const bool tabled = !ts.h_row0.empty();
    alloc_tiles(ts, tile, s.d, tabled ? (int)ts.h_row0.size() : (int)((s.n + tile - 1) / tile), st);
    if (ts.ntiles == 0) return;
    // lanes per row as in prep_rows; centroid [d] floats (rounded up to an even count) + per-group
    // partials (256 / kL groups x d x (8 + 4 + 4) bytes)
    const int L = s.d <= 16 ? 4 : s.d <= 32 ? 8 : 32;
    const size_t base = (size_t)((s.d + 1) & ~1) * sizeof(float);
    const size_t part = (size_t)(256 / L) * s.d * 16;
    const int warp_rows = base + part <= 200 * 1024 ? 1 : 0;
    const size_t smem = base + (warp_rows ? part : 0);
    auto run = [&](auto kern) {
        if (smem > 48 * 1024) TJ_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        launch(kern, ts.ntiles, 256, smem, st, s.src, s.dtype, s.n, s.d, tile, ts.ntiles, s.perm.p, s.nrm2.p,
               s.nrm2f.p, s.zn.p, s.en.p, s.yn.p, s.zl.p, ts.ctrT.p, ts.loT.p, ts.hiT.p, ts.rad.p, ts.maxZ.p,
               ts.maxE.p, ts.maxY.p, ts.maxB.p, ts.beta.p, ts.maxZl.p, ts.nvalid.p, ts.row0.p,
               tabled ? (const uint32_t*)ts.row0.p : (const uint32_t*)nullptr,
               tabled ? (const uint32_t*)ts.nvalid.p : (const uint32_t*)nullptr, warp_rows);
    };
    if (L == 4) run(tile_stats_kernel<4>);
    else if (L == 8) run(tile_stats_kernel<8>);
    else run(tile_stats_kernel<32>);
}

void gather_rows(const std::vector<const void*>& srcs, const std::vector<long long>& rows, int d, int esize,
                 void* dst, cudaStream_t st) {
    const int ns = (int)srcs.size();
    std::vector<long long> off(ns + 1, 0);
    for (int k = 0; k < ns; ++k) off[k + 1] = off[k] + rows[k];
    DBuf<const void*> dsrc((size_t)ns, st);
    DBuf<long long> doff((size_t)ns + 1, st);
    upload(dsrc.p, srcs.data(), ns * sizeof(void*), st);
    upload(doff.p, off.data(), (ns + 1) * sizeof(long long), st);
    const long long n = off[ns];
    if (n == 0) return;
    launch(gather_rows_kernel, (unsigned)((n + 7) / 8), 256, 0, st, (const void* const*)dsrc.p,
           (const long long*)doff.p, ns, n, d * esize, (uint8_t*)dst);
}

void compute_perm_local(Side& s, cudaStream_t st) {
    if (s.njc <= 1 || s.n == 0) {
        s.emit = s.perm.p;
        return;
    }
    s.perm_local = DBuf<uint32_t>((size_t)s.n, st);
    launch(perm_local_kernel, (unsigned)((s.n + 255) / 256), 256, 0, st, s.keys.p, s.perm.p, s.d_rowoff, s.n,
           s.perm_local.p);
    s.emit = s.perm_local.p;
}

void build_candidates(const TileSet& tr, const TileSet& ts, double Tp, bool self_join, int chunk_items,
                      Candidates& c, cudaStream_t st) {
    const int ntR = tr.ntiles, ntS = ts.ntiles, d = tr.d;
    const int words = (ntS + 31) / 32;
    c.cnt = DBuf<uint32_t>((size_t)std::max(ntR, 1), st);
    c.off = DBuf<uint32_t>((size_t)std::max(ntR, 1), st);
    c.dev_counts = DBuf<uint32_t>(2, st);
    TJ_CUDA(cudaMemsetAsync(c.dev_counts.p, 0, 2 * sizeof(uint32_t), st));
    const size_t maxc = (size_t)ntR * (size_t)ntS;
    c.jlist = DBuf<uint32_t>(std::max<size_t>(maxc, 1), st);
    c.chunks_cap = maxc / (size_t)chunk_items + (size_t)ntR + 1;
    c.chunks = DBuf<uint4>(c.chunks_cap, st);
    if (ntR == 0 || ntS == 0) return;
    DBuf<uint32_t> bitmap((size_t)ntR * words, st);
    TJ_CUDA(cudaMemsetAsync(bitmap.p, 0, bitmap.bytes(), st));
    const int ci = (size_t)3 * 16 * d * sizeof(float) <= 200 * 1024 ? 16 : (size_t)3 * 4 * d * sizeof(float) <= 200 * 1024 ? 4 : 1;
    const size_t smem = (size_t)3 * ci * d * sizeof(float);
    if (smem > 200 * 1024) fail(-7, "dimension too large for the candidate test");
    dim3 grid((unsigned)((ntS + 255) / 256), (unsigned)((ntR + ci - 1) / ci));
#define TJ_CAND(CI)                                                                                                 \
    TJ_CUDA(cudaFuncSetAttribute(cand_test<CI>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));          \
    launch(cand_test<CI>, grid, 256, smem, st, tr.ctrT.p, tr.loT.p, tr.hiT.p, tr.rad.p, ntR, ts.ctrT.p, ts.loT.p,      \
                                           ts.hiT.p, ts.rad.p, ntS, d, tr.tile, ts.tile, Tp, self_join ? 1 : 0,      \
                                           bitmap.p, words)
    if (ci == 16) { TJ_CAND(16); } else if (ci == 4) { TJ_CAND(4); } else { TJ_CAND(1); }
#undef TJ_CAND
    TJ_CUDA(cudaGetLastError());
    launch(cand_count, (unsigned)((ntR * 32 + 255) / 256), 256, 0, st, bitmap.p, words, ntR, c.cnt.p);
    DBuf<uint32_t> sws(scan_workspace_elems((size_t)ntR) + 4, st);
    exclusive_scan_u32(c.cnt.p, c.off.p, (size_t)ntR, c.dev_counts.p, sws.p, st);
    launch(cand_fill, (unsigned)((ntR * 32 + 255) / 256), 256, 0, st, bitmap.p, words, ntR, c.off.p, c.jlist.p,
           (const uint32_t*)nullptr);
    // chunks: (w, I) order so that concurrently running CTAs share the same S window
    DBuf<uint32_t> nch((size_t)ntR, st), cbase((size_t)ntR, st);
    launch(chunk_counts, (unsigned)((ntR + 255) / 256), 256, 0, st, c.cnt.p, ntR, chunk_items, nch.p);
    exclusive_scan_u32(nch.p, cbase.p, (size_t)ntR, c.dev_counts.p + 1, sws.p, st);
    const size_t cap = c.chunks_cap;
    DBuf<uint64_t> keys(cap, st), ktmp(cap, st);
    DBuf<uint32_t> vals(cap, st), vtmp(cap, st);
    launch(fill_keys_max, (unsigned)((cap + 255) / 256), 256, 0, st, keys.p, vals.p, 0, cap, c.dev_counts.p + 1);
    launch(chunk_keys, (unsigned)((ntR + 255) / 256), 256, 0, st, nch.p, cbase.p, ntR, cap, keys.p, vals.p);
    DBuf<uint32_t> rws(radix_workspace_elems(cap), st);
    radix_sort(keys.p, vals.p, ktmp.p, vtmp.p, cap, 48, rws.p, st);
    launch(chunk_emit, (unsigned)((cap + 255) / 256), 256, 0, st, keys.p, cap, c.dev_counts.p + 1, c.cnt.p, c.off.p,
                                                               chunk_items, c.chunks.p);
    TJ_CUDA(cudaGetLastError());
}

void half_masks(const std::vector<HalfView>& views, const Candidates& c, int ntR_total, const uint4* rtiles,
                const JoinParams* jps, bool self_join, cudaStream_t st) {
    if (ntR_total == 0 || views.empty()) return;
    int dmax = 1;
    for (const auto& v : views) dmax = std::max(dmax, v.d);
    DBuf<HalfView> dv(views.size(), st);
    upload(dv.p, views.data(), views.size() * sizeof(HalfView), st);
    const size_t smem = (size_t)8 * 3 * dmax * sizeof(float);   // one R tile per warp
    if (smem > 48 * 1024)
        TJ_CUDA(cudaFuncSetAttribute(half_mask_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    // warps stride over the chunks (their count is on the device); at most the chunk capacity
    const unsigned blocks = (unsigned)std::min<size_t>((size_t)num_sms() * 8, (c.chunks_cap + 7) / 8);
    launch(half_mask_kernel, std::max(1u, blocks), 256, smem, st, (const uint4*)c.chunks.p,
           (const uint32_t*)(c.dev_counts.p + 1), c.jlist.p, rtiles, jps, (const HalfView*)dv.p, self_join ? 1 : 0,
           dmax);
}

void tile_stats_rowmajor(TileSet& ts, cudaStream_t st) {
    const size_t n = (size_t)std::max(ts.ntiles, 1) * ts.d;
    ts.ctrR = DBuf<float>(n, st);
    ts.loR = DBuf<float>(n, st);
    ts.hiR = DBuf<float>(n, st);
    if (ts.ntiles == 0) return;
    const size_t m = (size_t)ts.ntiles * ts.d;
    launch(stats_rowmajor_kernel, (unsigned)((m + 255) / 256), 256, 0, st, (const float*)ts.ctrT.p,
           (const float*)ts.loT.p, (const float*)ts.hiT.p, ts.ntiles, ts.d, ts.ctrR.p, ts.loR.p, ts.hiR.p);
}

void build_candidates_batched(const std::vector<CandClassView>& classes, const std::vector<CandBlock>& blocks,
                              const std::vector<double>& Tp_per_block, int ntR_total, int words, int chunk_items,
                              const std::vector<uint32_t>& rtile_sbase, Candidates& c, cudaStream_t st) {
    const int ntR = ntR_total;
    const int nb = (int)blocks.size();
    c.cnt = DBuf<uint32_t>((size_t)std::max(ntR, 1), st);
    c.off = DBuf<uint32_t>((size_t)std::max(ntR, 1), st);
    c.dev_counts = DBuf<uint32_t>(2, st);
    TJ_CUDA(cudaMemsetAsync(c.dev_counts.p, 0, 2 * sizeof(uint32_t), st));
    size_t maxc = 0;
    for (const auto& b : blocks) maxc += (size_t)b.ni * b.nj;
    c.jlist = DBuf<uint32_t>(std::max<size_t>(maxc, 1), st);
    c.chunks_cap = maxc / (size_t)chunk_items + (size_t)ntR + 1;
    c.chunks = DBuf<uint4>(c.chunks_cap, st);
    if (ntR == 0 || nb == 0) return;
    int dmax = 1;
    for (const auto& v : classes) dmax = std::max(dmax, v.d);
    DBuf<CandBlock> dblk((size_t)nb, st);
    DBuf<CandClassView> dview(classes.size(), st);
    DBuf<double> dtp((size_t)nb, st);
    DBuf<uint32_t> dsb((size_t)ntR, st);
    upload(dblk.p, blocks.data(), nb * sizeof(CandBlock), st);
    upload(dview.p, classes.data(), classes.size() * sizeof(CandClassView), st);
    upload(dtp.p, Tp_per_block.data(), nb * sizeof(double), st);
    upload(dsb.p, rtile_sbase.data(), ntR * sizeof(uint32_t), st);
    DBuf<uint32_t> bitmap((size_t)ntR * words, st);
    TJ_CUDA(cudaMemsetAsync(bitmap.p, 0, bitmap.bytes(), st));
    const size_t smem = (size_t)3 * 16 * dmax * sizeof(float);
    if (smem > 200 * 1024) fail(-7, "dimension too large for the batched candidate test");
    TJ_CUDA(cudaFuncSetAttribute(cand_test_batched<16>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    launch(cand_test_batched<16>, nb, 256, smem, st, (const CandBlock*)dblk.p, (const CandClassView*)dview.p,
           (const double*)dtp.p, bitmap.p, words);
    launch(cand_count, (unsigned)((ntR * 32 + 255) / 256), 256, 0, st, bitmap.p, words, ntR, c.cnt.p);
    DBuf<uint32_t> sws(scan_workspace_elems((size_t)ntR) + 4, st);
    exclusive_scan_u32(c.cnt.p, c.off.p, (size_t)ntR, c.dev_counts.p, sws.p, st);
    launch(cand_fill, (unsigned)((ntR * 32 + 255) / 256), 256, 0, st, bitmap.p, words, ntR, c.off.p, c.jlist.p,
           (const uint32_t*)dsb.p);
    DBuf<uint32_t> nch((size_t)ntR, st), cbase((size_t)ntR, st);
    launch(chunk_counts, (unsigned)((ntR + 255) / 256), 256, 0, st, c.cnt.p, ntR, chunk_items, nch.p);
    exclusive_scan_u32(nch.p, cbase.p, (size_t)ntR, c.dev_counts.p + 1, sws.p, st);
    const size_t cap = c.chunks_cap;
    DBuf<uint64_t> keys(cap, st), ktmp(cap, st);
    DBuf<uint32_t> vals(cap, st), vtmp(cap, st);
    launch(fill_keys_max, (unsigned)((cap + 255) / 256), 256, 0, st, keys.p, vals.p, (size_t)0, cap,
           (const uint32_t*)(c.dev_counts.p + 1));
    launch(chunk_keys, (unsigned)((ntR + 255) / 256), 256, 0, st, nch.p, cbase.p, ntR, cap, keys.p, vals.p);
    DBuf<uint32_t> rws(radix_workspace_elems(cap), st);
    radix_sort(keys.p, vals.p, ktmp.p, vtmp.p, cap, 48, rws.p, st);
    launch(chunk_emit, (unsigned)((cap + 255) / 256), 256, 0, st, keys.p, cap, (const uint32_t*)(c.dev_counts.p + 1),
           c.cnt.p, c.off.p, chunk_items, c.chunks.p);
}

}  // namespace tj
