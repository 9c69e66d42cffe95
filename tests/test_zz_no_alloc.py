"""The allocation-free sort entry point, called through the C ABI.

tj_sort_keys_noalloc exists for callers that cannot allocate device memory where
they need pairs in canonical order (a fixed arena owned by the host engine, HBM
held by another allocator, or no allocation latency allowed between launches).
It must give exactly the order the allocating path gives: here the canonical keys
returned by tj_join / tj_result_keys are shuffled on the device and sorted again
with the allocation-free entry point, twice in a row on the same shared scratch,
and both outputs must equal the join's keys bit for bit (integer keys, zero
tolerance).  This file is collected last on purpose.
"""
import ctypes as C

import numpy as np
import pytest
import torch

import tensorjoin_variants_b200 as tj
from tensorjoin_variants_b200 import _lib
from tensorjoin_variants_b200 import workloads as W

pytestmark = pytest.mark.gpu
MAX_KEYS = 1 << 20


def _bits(max_value: int) -> int:
    return max(1, int(max_value).bit_length())


def _noalloc_sort(keys_in: torch.Tensor, keys_out: torch.Tensor, n: int, bits: int) -> int:
    return _lib.lib().tj_sort_keys_noalloc(C.c_void_p(keys_in.data_ptr()), C.c_void_p(keys_out.data_ptr()),
                                           n, bits, C.c_void_p(torch.cuda.current_stream().cuda_stream))


def test_noalloc_sort_matches_join_keys_twice():
    w = W.uniform16(n=6000)
    X = torch.from_numpy(w.R).cuda()
    res = tj.join_result(X, None, eps2=w.T, mode="directed", screen="bf16")
    want = res.keys()                      # existing entry point: sorted canonical keys
    n = want.numel()
    assert 0 < n <= MAX_KEYS
    bits = _bits(6000 * 6000)
    g = torch.Generator(device="cuda").manual_seed(5)
    for _ in range(2):                     # two calls in a row share (and reuse) the static scratch
        shuffled = want[torch.randperm(n, device="cuda", generator=g)]
        out = torch.empty_like(shuffled)
        assert _noalloc_sort(shuffled, out, n, bits) == 0
        torch.cuda.synchronize()
        assert torch.equal(out, want)


def test_noalloc_sort_in_place_and_limits():
    rng = np.random.default_rng(9)
    keys = rng.integers(0, 1 << 40, size=200_000, dtype=np.int64)
    t = torch.from_numpy(keys).cuda()
    assert _noalloc_sort(t, t, t.numel(), 40) == 0   # in place
    torch.cuda.synchronize()
    assert np.array_equal(t.cpu().numpy(), np.sort(keys))
    big = torch.zeros(MAX_KEYS + 1, dtype=torch.int64, device="cuda")
    assert _noalloc_sort(big, big, MAX_KEYS + 1, 40) == -1   # beyond the stated maximum: rejected
    assert b"maximum" in _lib.lib().tj_last_error_string()
    # partly overlapping input and output ranges are rejected (the same array or disjoint ones only)
    assert _noalloc_sort(big[:1000], big[500:1500], 1000, 40) == -1
    assert b"overlap" in _lib.lib().tj_last_error_string()
    assert _noalloc_sort(big, big, 0, 40) == 0                # empty: nothing to do


@pytest.mark.parametrize("n", [1, 16384, 16385, MAX_KEYS])
def test_noalloc_sort_sizes(n):
    """The one-block path's limit (16,384 keys) on both sides, a single key, and exactly the maximum
    (the ping-pong buffer full, the histogram and scan area at its largest), out of place."""
    rng = np.random.default_rng(n)
    keys = rng.integers(0, 1 << 40, size=n, dtype=np.int64)
    t = torch.from_numpy(keys).cuda()
    out = torch.empty_like(t)
    assert _noalloc_sort(t, out, n, 40) == 0
    torch.cuda.synchronize()
    assert np.array_equal(out.cpu().numpy(), np.sort(keys))
    assert np.array_equal(t.cpu().numpy(), keys)   # the input is left as it was
