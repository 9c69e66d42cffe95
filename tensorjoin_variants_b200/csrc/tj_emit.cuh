// Warp-level emission of pair keys into global buffers (shared by every screen kernel).
//
// Each warp reserves a private chunk of a buffer with one atomicAdd and fills it over
// many batches; the unused tail of a chunk is padded with the sentinel key (all ones),
// which sorts after every valid key.  Slots at or beyond the capacity are counted but not
// written, so the host sees the overflow and reruns with larger buffers.  Compared with
// one atomic per pair (src/run_g2a_tensorjoin.py:109-132) this needs one global atomic per
// 256 slots per warp.
#pragma once

#include "tj_common.cuh"

namespace tj {

constexpr unsigned kEmitChunk = 256;

struct WarpAppender {
    unsigned long long base = 0;
    unsigned used = 0, size = 0;   // size == 0: no chunk reserved yet
    unsigned long long valid = 0;

    // Reserve `t` slots (warp-uniform total); returns the first slot of this batch.
    TJ_DEV unsigned long long reserve(unsigned t, unsigned long long* reserved, uint64_t* buf,
                                      unsigned long long cap) {
        if (used + t > size) {
            pad(buf, cap);
            const unsigned want = t > kEmitChunk ? t : kEmitChunk;
            unsigned long long b = 0;
            if (lane_id() == 0) b = atomicAdd(reserved, (unsigned long long)want);
            base = __shfl_sync(0xffffffffu, b, 0);
            used = 0;
            size = want;
        }
        const unsigned long long r = base + used;
        used += t;
        valid += t;
        return r;
    }
    // Fill the rest of the current chunk with sentinels (warp-collective).
    TJ_DEV void pad(uint64_t* buf, unsigned long long cap) {
        for (unsigned k = used + lane_id(); k < size; k += 32)
            if (base + k < cap) buf[base + k] = kSentinel;
        used = size;
    }
};

// Canonical key of a pair of original row ids: i * n_cols + j (self-join: lo * N + hi).
TJ_DEV uint64_t pair_key(const JoinParams& jp, uint32_t oi, uint32_t oj) {
    if (jp.self_join) {
        const uint32_t lo = oi < oj ? oi : oj, hi = oi < oj ? oj : oi;
        return jp.key_off + (uint64_t)lo * (uint64_t)jp.n_cols + hi;
    }
    return jp.key_off + (uint64_t)oi * (uint64_t)jp.n_cols + oj;
}

}  // namespace tj
