"""GPU: the single-sweep radix passes (arrays of more than 2^20 keys) inside real joins.

Three shapes reach them: the output sort of a join with millions of pairs (an odd pass count leaves
the result in the temporaries, which then become the result), the Morton sort with row ids of a
side of more than 2^20 rows, and the same sort over a class of packed joins (join number above the
Morton bits).  Each result is checked against the oracle or against a closed form.
"""
import numpy as np
import pytest
import torch

import oracle
import tensorjoin_variants_b200 as tj

pytestmark = pytest.mark.gpu


def _keys(res):
    return res.keys().cpu().numpy().view(np.uint64)


@pytest.mark.parametrize("screen", ["bf16", "plain"])
def test_output_sort_all_pairs(screen):
    """3,000 x 3,000 rows under a threshold that takes every pair: 9 M keys over 24 bits (three
    passes), which must come out as exactly 0, 1, ..., 9 M - 1."""
    g = np.random.default_rng(11)
    R = g.standard_normal((3000, 8)).astype(np.float32)
    S = g.standard_normal((3000, 8)).astype(np.float32)
    res = tj.join_result(torch.from_numpy(R).cuda(), torch.from_numpy(S).cuda(), eps2=1e6, screen=screen,
                         guards=True)
    k = _keys(res)
    assert len(k) == 9_000_000
    assert np.array_equal(k, np.arange(9_000_000, dtype=np.uint64))


def test_output_sort_directed_all_pairs():
    """Directed self-join of 1,500 rows taking every pair: 2.25 M keys after the expansion."""
    g = np.random.default_rng(12)
    X = g.standard_normal((1500, 4)).astype(np.float32)
    res = tj.join_result(torch.from_numpy(X).cuda(), None, eps2=1e6, mode="directed", screen="fp16", guards=True)
    assert np.array_equal(_keys(res), np.arange(1500 * 1500, dtype=np.uint64))


def test_index_sort_large_side():
    """1.2 M R rows (the Morton sort with row ids runs single-sweep) against 40 S rows."""
    g = np.random.default_rng(13)
    R = g.standard_normal((1_200_000, 4)).astype(np.float32)
    S = g.standard_normal((40, 4)).astype(np.float32)
    T = 0.05
    res = tj.join_result(torch.from_numpy(R).cuda(), torch.from_numpy(S).cuda(), eps2=T, screen="bf16x3",
                         guards=True)
    want = oracle.join_f32(R, S, T, "rs")
    assert len(want) > 1000
    assert np.array_equal(_keys(res), want)


@pytest.mark.parametrize("njoins", [200, 300])
def test_index_sort_packed_class(njoins):
    """Packed joins of 6,000 R rows each: one class of 1.2 M or 1.8 M rows whose Morton keys carry
    the join number above 32 Morton bits (40 or 41 bits: five or six passes)."""
    g = np.random.default_rng(14 + njoins)
    joins = []
    for _ in range(njoins):
        R = g.standard_normal((6000, 8)).astype(np.float32)
        S = g.standard_normal((32, 8)).astype(np.float32)
        joins.append((R, S, 1.2))
    out = tj.join_batched([(torch.from_numpy(R).cuda(), torch.from_numpy(S).cuda(), e) for R, S, e in joins],
                          screen="bf16x3", guards=True)
    for q in range(0, njoins, 37):
        R, S, e = joins[q]
        want = oracle.join_f32(R, S, e * e, "rs")
        i, j = out[q]
        got = (i.cpu().numpy().astype(np.uint64) * np.uint64(S.shape[0]) + j.cpu().numpy().astype(np.uint64))
        assert np.array_equal(got, want), q


def test_batched_host_views_of_one_array():
    """Joins whose rows are views of two pinned host arrays (one per side) move in one copy per array
    and come back as host pairs identical to the oracle's."""
    g = np.random.default_rng(21)
    nr = g.integers(50, 3000, 40)
    ns = g.integers(50, 3000, 40)
    RA = torch.from_numpy(g.standard_normal((int(nr.sum()), 16)).astype(np.float32)).pin_memory()
    SA = torch.from_numpy(g.standard_normal((int(ns.sum()), 16)).astype(np.float32)).pin_memory()
    ro, so = np.concatenate([[0], np.cumsum(nr)]), np.concatenate([[0], np.cumsum(ns)])
    joins = [(RA[ro[k]:ro[k + 1]], SA[so[k]:so[k + 1]], 2.0) for k in range(40)]
    out = tj.join_batched(joins, screen="bf16x3", guards=True)
    for k in range(40):
        R, S, e = joins[k]
        want = oracle.join_f32(R.numpy(), S.numpy(), e * e, "rs")
        i, j = out[k]
        assert not i.is_cuda
        got = i.numpy().astype(np.uint64) * np.uint64(S.shape[0]) + j.numpy().astype(np.uint64)
        assert np.array_equal(got, want), k
