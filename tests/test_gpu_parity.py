"""GPU parity: every path's pair set is bit-identical to the CPU oracle (same seeded inputs, same T).

The tolerance is zero: the pair set is discrete and the FP64 refinement uses the
oracle's summation order.  Pairs are compared as canonical uint64 keys.
"""
import ctypes as C
import hashlib
import json
from pathlib import Path

import numpy as np
import pytest
import torch

import oracle
import tensorjoin_variants_b200 as tj
from tensorjoin_variants_b200 import _lib
from tensorjoin_variants_b200 import workloads as W

pytestmark = pytest.mark.gpu
GOLDEN = Path(__file__).resolve().parent / "golden"
G = json.loads((GOLDEN / "golden.json").read_text())
FLOAT_SCREENS = ["plain", "bf16", "fp16", "bf16x3", "fp16x3"]


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a, dtype="<u8").tobytes()).hexdigest()


def gpu_keys(R, S, T, mode, screen, **kw):
    """Keys of one GPU join; every parity join runs with guard regions after its output buffers
    (an out-of-bounds write fails the join)."""
    Rt = torch.from_numpy(np.ascontiguousarray(R)).cuda()
    St = None if S is None else torch.from_numpy(np.ascontiguousarray(S)).cuda()
    kw.setdefault("guards", True)
    res = tj.join_result(Rt, St, eps2=T, mode=mode, screen=screen, **kw)
    k = res.keys().cpu().numpy().view(np.uint64)
    i, j = res.pairs()
    n_cols = R.shape[0] if S is None else S.shape[0]
    assert np.array_equal(i.cpu().numpy(), (k // np.uint64(n_cols)).astype(np.int64))
    assert np.array_equal(j.cpu().numpy(), (k % np.uint64(n_cols)).astype(np.int64))
    return k, res.stats


def oracle_keys(R, S, T, mode):
    return oracle.join_f32(R, S, T, mode)


def assert_same(got, want, label=""):
    if not np.array_equal(got, want):
        extra = np.setdiff1d(got, want)
        missing = np.setdiff1d(want, got)
        raise AssertionError(f"{label}: got {len(got)} want {len(want)}; extra {extra[:10]} missing {missing[:10]}")


@pytest.mark.parametrize("screen", FLOAT_SCREENS)
def test_uniform16_full_config(screen):
    """Config 1 at full size (20,000 x 16, ~32 neighbours, i < j) against the pinned golden hash."""
    w = W.uniform16()
    k, st = gpu_keys(w.R, None, w.T, "upper", screen)
    assert len(k) == G["uniform16"]["oracle_upper_count"]
    assert sha(k) == G["uniform16"]["oracle_upper_sha256"]
    assert st["result_pairs"] == len(k)


@pytest.mark.parametrize("screen", FLOAT_SCREENS)
def test_gds_fixture_directed(screen):
    """GDS-Join's 100,000-point 2-D test set at eps = 1.0 (directed, self pairs included)."""
    X = np.load(GOLDEN / "gds_test_dat_f32.npy")
    g = G["gds_test_dat"]
    k, _ = gpu_keys(X, None, 1.0, "directed", screen)
    assert len(k) == g["oracle_directed_count"]
    assert sha(k) == g["oracle_directed_sha256"]


@pytest.mark.parametrize("screen", FLOAT_SCREENS)
def test_mixture_rs_small(screen):
    w = W.mixture64(n=6000, samples=1 << 16, screen=screen)
    k, st = gpu_keys(w.R, w.S, w.T, "rs", screen)
    assert_same(k, oracle_keys(w.R, w.S, w.T, "rs"), screen)
    assert st["pairs_screened"] <= w.candidate_pairs_all
    if screen == "bf16x3":   # centred hi/lo operands keep the certified band narrow on clustered data
        assert st["band"] <= 0.01 * st["pairs_screened"]


@pytest.mark.parametrize("screen", FLOAT_SCREENS)
def test_factor512_small(screen):
    w = W.factor512(n=3000, samples=1 << 16)
    k, st = gpu_keys(w.R, w.S, w.T, "rs", screen)
    assert_same(k, oracle_keys(w.R, w.S, w.T, "rs"), screen)
    assert st["band"] >= 0


@pytest.mark.parametrize("screen", FLOAT_SCREENS)
@pytest.mark.parametrize("d", [1, 3, 8, 16, 17, 31, 32, 33, 63, 65, 130])
def test_ragged_dimensions(screen, d):
    rng = np.random.default_rng(100 + d)
    R = rng.standard_normal((700, d)).astype(np.float32)
    S = rng.standard_normal((900, d)).astype(np.float32)
    T = float(np.quantile(((R[:50, None, :] - S[None, :200, :]) ** 2).sum(-1), 0.01))
    k, _ = gpu_keys(R, S, T, "rs", screen)
    assert_same(k, oracle_keys(R, S, T, "rs"), f"{screen} d={d}")


@pytest.mark.parametrize("screen", FLOAT_SCREENS)
def test_self_join_modes(screen):
    rng = np.random.default_rng(21)
    X = rng.random((2500, 24)).astype(np.float32)
    X[2000:2100] = X[:100]            # exact duplicates: d2 == 0
    T = 0.35
    for mode in ("upper", "directed"):
        k, _ = gpu_keys(X, None, T, mode, screen)
        assert_same(k, oracle_keys(X, None, T, mode), f"{screen} {mode}")


@pytest.mark.parametrize("screen", FLOAT_SCREENS)
def test_edge_cases(screen):
    rng = np.random.default_rng(22)
    one = rng.random((1, 8)).astype(np.float32)
    many = rng.random((300, 8)).astype(np.float32)
    # single row against many, and many against a single row
    assert_same(gpu_keys(one, many, 0.5, "rs", screen)[0], oracle_keys(one, many, 0.5, "rs"))
    assert_same(gpu_keys(many, one, 0.5, "rs", screen)[0], oracle_keys(many, one, 0.5, "rs"))
    # eps = 0: only exact duplicates
    dup = np.concatenate([many, many[:37]])
    assert_same(gpu_keys(dup, None, 0.0, "upper", screen)[0], oracle_keys(dup, None, 0.0, "upper"))
    # all-zero input at a tiny eps accepts every pair; +-1 blocks at eps = 0 give the two sign blocks
    Z = np.zeros((300, 32), np.float32)
    assert len(gpu_keys(Z, None, 2.0 ** -40, "directed", screen)[0]) == 300 * 300
    P = np.concatenate([np.ones((130, 64), np.float32), -np.ones((140, 64), np.float32)])
    kp, _ = gpu_keys(P, None, 0.0, "directed", screen)
    assert_same(kp, oracle_keys(P, None, 0.0, "directed"))


def test_empty_inputs():
    R = torch.zeros((0, 16), device="cuda")
    S = torch.rand((10, 16), device="cuda")
    i, j = tj.join(R, S, 0.5)
    assert i.numel() == 0 and j.numel() == 0
    i, j = tj.join(S, R, 0.5)
    assert i.numel() == 0


def test_capacity_retry():
    """A tiny initial capacity forces the overflow-and-retry pass; the result must not change."""
    w = W.uniform16(n=4000)
    want = oracle_keys(w.R, None, w.T, "upper")
    for screen in FLOAT_SCREENS:
        k, st = gpu_keys(w.R, None, w.T, "upper", screen, capacity=512)
        assert st["retries"] >= 1
        assert_same(k, want, screen)


def test_bad_inputs_fail_closed():
    X = torch.rand((500, 16), device="cuda")
    X[17, 3] = float("nan")
    with pytest.raises(_lib.TJError) as e:
        tj.self_join(X, 0.3)
    assert e.value.code == -3
    Y = torch.rand((500, 16), device="cuda") * 1e5
    Y[:250] -= 2e5                   # centred values still beyond the FP16 range
    for scr in ("fp16", "fp16x3"):
        with pytest.raises(_lib.TJError) as e:
            tj.self_join(Y, 0.3, screen=scr)
        assert e.value.code == -4
    F = torch.rand((10, 4), device="cuda")
    with pytest.raises(_lib.TJError) as e:   # the int8-limb screen takes int14 data only
        tj.join_result(F, F, 0.1, mode="rs", screen="int8limb")
    assert e.value.code == -7


@pytest.mark.parametrize("screen", ["bf16", "fp16", "bf16x3"])
def test_metamorphic(screen):
    rng = np.random.default_rng(23)
    R = rng.standard_normal((1500, 40)).astype(np.float32)
    S = rng.standard_normal((1700, 40)).astype(np.float32)
    T = 40.0
    base, _ = gpu_keys(R, S, T, "rs", screen)
    assert_same(base, oracle_keys(R, S, T, "rs"))
    assert_same(gpu_keys(-R, -S, T, "rs", screen)[0], base, "negate")
    sc = np.float32(2.0 ** 8)
    assert_same(gpu_keys(R * sc, S * sc, T * 2.0 ** 16, "rs", screen)[0], base, "scale")
    perm = rng.permutation(40)
    sign = np.where(rng.random(40) < 0.5, -1, 1).astype(np.float32)
    assert_same(gpu_keys(R[:, perm] * sign, S[:, perm] * sign, T, "rs", screen)[0], base, "dims")
    rp = rng.permutation(1500)
    kp, _ = gpu_keys(R[rp], S, T, "rs", screen)
    inv = np.argsort(rp)
    i, j = oracle.keys_to_ij(kp, 1700)
    remapped = np.sort(rp[i].astype(np.uint64) * np.uint64(1700) + j.astype(np.uint64))
    assert_same(remapped, base, "row permutation")
    assert len(inv) == 1500


def test_host_arrays_roundtrip():
    """Host (numpy) inputs: copied in, joined on the GPU, results returned on the host."""
    w = W.uniform16(n=3000)
    i, j = tj.self_join(w.R, w.eps)
    assert isinstance(i, torch.Tensor) and not i.is_cuda
    k = i.numpy().astype(np.uint64) * np.uint64(3000) + j.numpy().astype(np.uint64)
    assert_same(k, oracle_keys(w.R, None, w.eps * w.eps, "upper"))


def test_neighbor_table_matches_pairs():
    w = W.uniform16(n=3000)
    res = tj.join_result(torch.from_numpy(w.R).cuda(), None, eps2=w.T, mode="directed")
    counts, flat = res.neighbor_table()
    i, j = res.pairs()
    assert int(counts.sum()) == res.count
    assert torch.equal(torch.bincount(i, minlength=3000).to(torch.int32), counts)
    assert torch.equal(flat, j)


@pytest.mark.parametrize("n", [20000, 140000])   # 140,000 rows: principal-direction cells
def test_index_structure(n):
    w = W.mixture64(n=n, samples=1 << 14)
    idx = tj.build_index(torch.from_numpy(w.R).cuda(), w.eps)
    perm = idx.perm.cpu().numpy()
    assert np.array_equal(np.sort(perm), np.arange(n))
    keys = idx.keys.cpu().numpy()
    assert np.all(keys[1:] >= keys[:-1])
    cs = idx.cell_start.cpu().numpy()
    assert cs[0] == 0 and cs[-1] == n and np.all(np.diff(cs) > 0)
    assert np.all(keys[cs[:-1]][1:] != keys[cs[:-1]][:-1])
    tp = idx.tile_pairs.cpu().numpy()
    assert tp.shape[1] == 2 and len(tp) >= idx.n_tiles // 2


# ---------------------------------------------------------------- int14 data, exact int8-limb screen
@pytest.mark.parametrize("four", [False, True])
@pytest.mark.parametrize("d", [128, 100, 200, 300])
def test_int14_self_join_exact(d, four):
    """Both int8-limb screens (high-limb product + exact integer band refinement, or all four limb
    products decided in the kernel) against the exact integer oracle; d = 300 exceeds the high-limb
    screen's resident R tile, so it takes the four-product screen either way."""
    w = W.int14x128(n=5000, d=d, samples=1 << 14)
    for mode in ("upper", "directed"):
        want = oracle.join_i16(w.R, None, w.T, mode)
        k, st = gpu_keys(w.R, None, w.T, mode, "int8limb", i8_four_products=four)
        assert_same(k, want, f"d={d} {mode} four={four}")
        if four or d > 256:
            assert st["band"] == 0
        assert st["screen_ops_issued"] > 0
        # the full-size int14 join takes principal-direction cells (2M rows): same pairs here
        k, st = gpu_keys(w.R, None, w.T, mode, "int8limb", index_frame="pca", i8_four_products=four)
        assert_same(k, want, f"d={d} {mode} pca four={four}")
        assert st["index_frame"] == (1 if d <= 128 else 0)   # principal directions up to d = 128


@pytest.mark.parametrize("four", [False, True])
def test_int14_rs_ties_and_extremes(four):
    rng = np.random.default_rng(31)
    R = rng.integers(-8192, 8192, size=(1500, 128), dtype=np.int16)
    S = rng.integers(-8192, 8192, size=(1700, 128), dtype=np.int16)
    R[:8] = 8191
    S[:8] = -8192
    R[8:16] = -8192
    S[8:16] = 8191
    S[100:150] = R[200:250] + rng.integers(-1, 2, size=(50, 128)).astype(np.int16)
    S[100:150] = np.clip(S[100:150], -8192, 8191)
    d2 = ((R[200:250].astype(np.int64) - S[100:150].astype(np.int64)) ** 2).sum(1)
    T = int(np.median(d2))      # several pairs sit exactly on the threshold
    assert np.count_nonzero(d2 == T) >= 1
    k, st = gpu_keys(R, S, T, "rs", "int8limb", i8_four_products=four)
    assert_same(k, oracle.join_i16(R, S, T, "rs"), "ties")
    # the largest possible distance (all +8191 vs all -8192) decides exactly at its own value
    Tmax = 128 * (8191 + 8192) ** 2
    kx, _ = gpu_keys(R[:16], S[:16], Tmax, "rs", "int8limb", i8_four_products=four)
    assert_same(kx, oracle.join_i16(R[:16], S[:16], Tmax, "rs"), "extremes")
    kx2, _ = gpu_keys(R[:16], S[:16], Tmax - 1, "rs", "int8limb", i8_four_products=four)
    assert_same(kx2, oracle.join_i16(R[:16], S[:16], Tmax - 1, "rs"), "extremes-1")
    # a threshold far above every distance (2^61) accepts every pair; 0 accepts exact duplicates only
    kh, _ = gpu_keys(R[:300], S[:200], 1 << 61, "rs", "int8limb", i8_four_products=four)
    assert len(kh) == 300 * 200
    S0 = S.copy()
    S0[5] = R[7]
    k0, _ = gpu_keys(R, S0, 0, "rs", "int8limb", i8_four_products=four)
    assert_same(k0, oracle.join_i16(R, S0, 0, "rs"), "T = 0")


def test_int14_rejects_out_of_range_and_fraction():
    X = torch.full((300, 128), 9000, dtype=torch.int16, device="cuda")
    with pytest.raises(_lib.TJError) as e:
        tj.self_join(X, eps2=10, screen="int8limb")
    assert e.value.code == -3
    Y = torch.zeros((300, 128), dtype=torch.int16, device="cuda")
    with pytest.raises(_lib.TJError) as e:
        tj.self_join(Y, eps2=10.5, screen="int8limb")
    assert e.value.code == -1


# ---------------------------------------------------------------- batched ragged joins (one persistent screen launch)
def _ragged(njoins, seed, dims=(8, 32, 128), lo=50, hi=3000):
    rng = np.random.default_rng(seed)
    joins = []
    for k in range(njoins):
        nr = int(np.exp(rng.uniform(np.log(lo), np.log(hi))))
        ns = int(np.exp(rng.uniform(np.log(lo), np.log(hi))))
        d = int(rng.choice(dims))
        centres = rng.random((8, d))
        R = (centres[rng.integers(0, 8, nr)] + rng.standard_normal((nr, d)) * 0.05).astype(np.float32)
        S = (centres[rng.integers(0, 8, ns)] + rng.standard_normal((ns, d)) * 0.05).astype(np.float32)
        T = W.ragged_eps2(ns, d, 8, 0.05, 16)
        joins.append((R, S, T))
    return joins


@pytest.mark.parametrize("screen", ["bf16x3", "fp16", "plain"])
def test_batched_ragged_exact(screen):
    joins = _ragged(40, 41)
    joins.append((joins[0][0][:0], joins[1][1], 0.5))          # empty R side
    joins.append((joins[2][0], joins[3][1][:1], joins[3][2]))  # single S row (d may differ: reuse S of same d)
    joins[-1] = (joins[3][0], joins[3][1][:1], joins[3][2])
    dev = [(torch.from_numpy(R).cuda(), torch.from_numpy(S).cuda(), float(np.sqrt(T))) for R, S, T in joins]
    out = tj.join_batched(dev, screen=screen)
    assert len(out) == len(joins)
    for k, ((R, S, T), (i, j)) in enumerate(zip(joins, out)):
        Tk = float(np.sqrt(T)) ** 2
        want = oracle.join_f32(R, S, Tk, "rs") if len(R) and len(S) else np.empty(0, np.uint64)
        got = i.cpu().numpy().astype(np.uint64) * np.uint64(max(len(S), 1)) + j.cpu().numpy().astype(np.uint64)
        assert_same(got, want, f"{screen} join {k} d={R.shape[1]} {len(R)}x{len(S)}")


def test_batched_equals_single_joins():
    joins = _ragged(12, 42, dims=(32,))
    dev = [(torch.from_numpy(R).cuda(), torch.from_numpy(S).cuda(), float(np.sqrt(T))) for R, S, T in joins]
    out = tj.join_batched(dev, screen="bf16x3")
    for (Rt, St, e), (i, j) in zip(dev, out):
        i1, j1 = tj.join(Rt, St, e, screen="bf16x3")
        assert torch.equal(i, i1) and torch.equal(j, j1)


@pytest.mark.parametrize("screen", ["bf16", "fp16", "bf16x3", "fp16x3"])
def test_screen_error_within_certified_radius(screen):
    """Sampled tensor-core accumulators: the distance estimate's error against sequential FP64 stays
    inside the certified radius (the accumulation premise holds on these inputs), and the result is
    unchanged by the diagnostic pass."""
    for w in (W.factor512(n=4000, samples=1 << 15), W.mixture64(n=8000, samples=1 << 15),
              W.mixture64(n=8000, d=32, samples=1 << 15), W.mixture64(n=8000, d=8, samples=1 << 15)):
        R, S = torch.from_numpy(w.R).cuda(), torch.from_numpy(w.S).cuda()
        res = tj.join_result(R, S, eps2=w.T, screen=screen, screen_diag=True)
        st = res.stats
        assert st["screen_err_pairs"] > 0
        assert 0.0 < st["screen_err_over_bound"] < 1.0, st
        k = res.keys().cpu().numpy().view(np.uint64)
        assert_same(k, oracle_keys(w.R, w.S, w.T, "rs"), screen)


def test_threshold_ties_float():
    """T equal to the oracle's exact distance of chosen pairs: those pairs are in, nothing else changes."""
    rng = np.random.default_rng(51)
    R = rng.standard_normal((600, 64)).astype(np.float32)
    S = rng.standard_normal((700, 64)).astype(np.float32)
    ii = rng.integers(0, 600, 6)
    jj = rng.integers(0, 700, 6)
    for T in oracle.pair_d2(R, S, ii, jj):
        for screen in ("bf16", "fp16x3", "plain"):
            k, _ = gpu_keys(R, S, float(T), "rs", screen)
            assert_same(k, oracle_keys(R, S, float(T), "rs"), f"tie {screen}")


@pytest.mark.parametrize("screen", ["bf16x3", "plain"])
def test_batched_views_of_one_array(screen):
    """Joins given as back-to-back views of one device array per side (used in place, no gather)
    give the same pairs as the same joins in separate arrays; a partly adjacent batch is gathered."""
    joins = _ragged(16, 43, dims=(8, 32))
    by_d = {}
    for R, S, T in joins:
        by_d.setdefault(R.shape[1], []).append((R, S, T))
    views, separate = [], []
    for d, js in by_d.items():
        Rall = torch.from_numpy(np.concatenate([R for R, _, _ in js])).cuda()
        Sall = torch.from_numpy(np.concatenate([S for _, S, _ in js])).cuda()
        r0 = s0 = 0
        for R, S, T in js:
            views.append((Rall[r0:r0 + len(R)], Sall[s0:s0 + len(S)], float(np.sqrt(T))))
            separate.append((torch.from_numpy(R).cuda(), torch.from_numpy(S).cuda(), float(np.sqrt(T))))
            r0 += len(R)
            s0 += len(S)
    a = tj.join_batched(views, screen=screen)
    b = tj.join_batched(separate, screen=screen)
    mixed = [views[0], separate[1]] + views[2:]
    c = tj.join_batched(mixed, screen=screen)
    for (i, j), (i2, j2), (i3, j3) in zip(a, b, c):
        assert torch.equal(i, i2) and torch.equal(j, j2)
        assert torch.equal(i, i3) and torch.equal(j, j3)


def test_pool_usage_and_reserve():
    """The memory-pool entry points report sizes and grow the pool on request."""
    L = _lib.lib()
    r0, u0, h0 = C.c_int64(), C.c_int64(), C.c_int64()
    assert L.tj_pool_usage(C.byref(r0), C.byref(u0), C.byref(h0)) == 0
    want = r0.value + (256 << 20)
    assert L.tj_pool_reserve(want, C.c_void_p(torch.cuda.current_stream().cuda_stream)) == 0
    r1 = C.c_int64()
    assert L.tj_pool_usage(C.byref(r1), None, None) == 0
    assert r1.value >= want
    assert L.tj_pool_trim(0) == 0
    assert L.tj_pool_reserve(-1, None) != 0


def test_results_alive_across_joins_and_sizes():
    """Results held while later joins of other sizes run (workspace growth, result-buffer reuse)
    keep their pairs; a freed result's buffer handed to a later join does not disturb it."""
    ws = [W.mixture64(n=n, d=d, samples=1 << 14) for n, d in ((3000, 16), (12000, 64), (1500, 32))]
    ws.append(ws[1])
    want = [oracle_keys(w.R, w.S, w.T, "rs") for w in ws[:3]]
    want.append(want[1])
    held = []
    for k, w in enumerate(ws):
        res = tj.join_result(torch.from_numpy(w.R).cuda(), torch.from_numpy(w.S).cuda(), eps2=w.T, screen="bf16x3")
        held.append(res)
        if k == 1:
            held[0] = None   # release the first result while others stay alive
    for k in (1, 2, 3):
        assert_same(held[k].keys().cpu().numpy().view(np.uint64), want[k], f"held {k}")


def test_concurrent_host_threads():
    """Two host threads joining at once on their own streams (one workspace per thread)."""
    import threading
    ws = [W.mixture64(n=6000, d=32, seed=s, samples=1 << 14) for s in (11, 12)]
    want = [oracle_keys(w.R, w.S, w.T, "rs") for w in ws]
    out = [None, None]
    errs = []

    def run(k):
        try:
            s = torch.cuda.Stream()
            with torch.cuda.stream(s):
                R, S = torch.from_numpy(ws[k].R).cuda(), torch.from_numpy(ws[k].S).cuda()
                for _ in range(3):
                    res = tj.join_result(R, S, eps2=ws[k].T, screen="bf16x3")
                    out[k] = res.keys().cpu().numpy().view(np.uint64)
        except Exception as e:   # surfaced below
            errs.append(e)

    th = [threading.Thread(target=run, args=(k,)) for k in (0, 1)]
    for t in th:
        t.start()
    for t in th:
        t.join()
    assert not errs, errs
    for k in (0, 1):
        assert_same(out[k], want[k], f"thread {k}")


@pytest.mark.parametrize("screen", ["fp16", "bf16"])
@pytest.mark.parametrize("shape", [(2000, 1500, 512), (300, 700, 256), (1100, 257, 320)])
def test_cta_pair_screen(screen, shape):
    """The CTA-pair screen (cta_group::2, 256 x 256 tiles over two SMs) gives the oracle's pairs,
    including an odd number of 128-row R tiles and S sides that are not a multiple of 256 rows."""
    nr, ns, d = shape
    rng = np.random.default_rng(nr + ns + d)
    R = (rng.standard_normal((nr, d)) / np.sqrt(d)).astype(np.float32)
    S = (rng.standard_normal((ns, d)) / np.sqrt(d)).astype(np.float32)
    T = float(np.quantile(((R[:60, None, :].astype(np.float64) - S[None, :300, :]) ** 2).sum(-1), 0.01))
    want = oracle_keys(R, S, T, "rs")
    Rt, St = torch.from_numpy(R).cuda(), torch.from_numpy(S).cuda()
    res = tj.join_result(Rt, St, eps2=T, screen=screen)
    assert res.stats["screen_pair"] == 1, res.stats
    assert_same(res.keys().cpu().numpy().view(np.uint64), want, f"pair {screen} {shape}")
    one = tj.join_result(Rt, St, eps2=T, screen=screen, cta_pair=False)
    assert one.stats["screen_pair"] == 0
    assert_same(one.keys().cpu().numpy().view(np.uint64), want, f"one-SM {screen} {shape}")


_PCA_CASE = {}


def _pca_case():
    """2,000 x 130,000 rows of the 64-d mixture: 132,000 rows in all, enough for the automatic
    principal-direction index frame (the oracle takes a few seconds; computed once)."""
    if not _PCA_CASE:
        w = W.mixture64(n=130000, samples=1 << 14)
        R = np.ascontiguousarray(w.R[:2000])
        _PCA_CASE.update(R=R, S=w.S, T=w.T, want=oracle_keys(R, w.S, w.T, "rs"))
    return _PCA_CASE


@pytest.mark.parametrize("screen", ["plain", "fp16", "bf16x3"])
def test_principal_direction_frame_auto(screen):
    """A single join with enough rows picks the principal-direction cells; the pairs stay the
    oracle's, and forcing the input-dimension cells gives the same pairs."""
    c = _pca_case()
    k, st = gpu_keys(c["R"], c["S"], c["T"], "rs", screen)
    assert st["index_frame"] == 1, st
    assert_same(k, c["want"], f"pca {screen}")
    k2, st2 = gpu_keys(c["R"], c["S"], c["T"], "rs", screen, index_frame="axes")
    assert st2["index_frame"] == 0
    assert_same(k2, c["want"], f"axes {screen}")
    small = W.mixture64(n=6000, samples=1 << 14)   # below the row threshold: input-dimension cells
    _, st3 = gpu_keys(small.R, small.S, small.T, "rs", screen)
    assert st3["index_frame"] == 0


@pytest.mark.parametrize("screen", FLOAT_SCREENS)
@pytest.mark.parametrize("d", [9, 16, 33, 64, 128])
def test_principal_direction_frame_forced(screen, d):
    """index_frame="pca" at small sizes, R-S and both self-join modes, against the oracle."""
    rng = np.random.default_rng(300 + d)
    centres = rng.random((6, d))
    R = (centres[rng.integers(0, 6, 1500)] + 0.05 * rng.standard_normal((1500, d))).astype(np.float32)
    S = (centres[rng.integers(0, 6, 2300)] + 0.05 * rng.standard_normal((2300, d))).astype(np.float32)
    T = float(np.quantile(((R[:60, None, :].astype(np.float64) - S[None, :400, :]) ** 2).sum(-1), 0.02))
    k, st = gpu_keys(R, S, T, "rs", screen, index_frame="pca")
    assert st["index_frame"] == 1
    assert_same(k, oracle_keys(R, S, T, "rs"), f"pca rs {screen} d={d}")
    for mode in ("upper", "directed"):
        k, st = gpu_keys(S, None, T, mode, screen, index_frame="pca")
        assert st["index_frame"] == 1
        assert_same(k, oracle_keys(S, None, T, mode), f"pca {mode} {screen} d={d}")


def test_frame_flags_exclusive():
    """Both frame flags at once is an invalid argument (rejected before any device work)."""
    R = torch.rand(300, 16, device="cuda")
    with pytest.raises(ValueError):
        tj.join_result(R, R, eps2=0.1, index_frame="both")
    opt = _lib.Options(0, 0, _lib.FLAG_FRAME_AXES | _lib.FLAG_FRAME_PCA)
    h = C.c_void_p()
    rc = _lib.lib().tj_join(C.c_void_p(R.data_ptr()), 300, C.c_void_p(R.data_ptr()), 300, 16, _lib.DTYPE["f32"],
                            0.1, _lib.MODE["rs"], _lib.SCREEN["bf16"], C.byref(opt), C.byref(h), None)
    assert rc != 0 and not h.value


@pytest.mark.parametrize("screen", ["bf16", "fp16", "bf16x3", "fp16x3"])
def test_fp32_band_stage(screen):
    """The certified FP32 band stage decides most band pairs without FP64 and changes no pair:
    R-S and both self-join modes, several d, ties at the threshold."""
    cases = []
    w = W.mixture64(n=6000, samples=1 << 14)
    cases.append((w.R, w.S, w.T, "rs"))
    f = W.factor512(n=2500, samples=1 << 14)
    cases.append((f.R, f.S, f.T, "rs"))
    rng = np.random.default_rng(77)
    for d in (3, 17, 130):
        X = rng.standard_normal((1800, d)).astype(np.float32)
        X[1500:1600] = X[:100]                      # d2 == 0 pairs
        T = float(np.quantile(((X[:50, None, :].astype(np.float64) - X[None, 50:400, :]) ** 2).sum(-1), 0.01))
        cases.append((X, None, T, "upper"))
        cases.append((X, None, T, "directed"))
    for R, S, T, mode in cases:
        want = oracle_keys(R, S, T, mode)
        k0, st0 = gpu_keys(R, S, T, mode, screen)
        k1, st1 = gpu_keys(R, S, T, mode, screen, band_fp32=True)
        label = f"{screen} {mode} d={R.shape[1]}"
        assert_same(k0, want, label + " fp64-only")
        assert_same(k1, want, label + " fp32 stage")
        assert st0["band_fp64"] == st0["band"], st0
        assert st1["band_fp64"] <= st1["band"], st1


def test_fp32_band_stage_batched():
    joins = _ragged(24, 43)
    dev = [(torch.from_numpy(R).cuda(), torch.from_numpy(S).cuda(), float(np.sqrt(T))) for R, S, T in joins]
    res = tj.join_batched_result(dev, screen="bf16", band_fp32=True)
    assert res.stats["band_fp64"] <= res.stats["band"]
    for k, ((R, S, T), (i, j)) in enumerate(zip(joins, res.split())):
        Tk = float(np.sqrt(T)) ** 2
        want = oracle.join_f32(R, S, Tk, "rs") if len(R) and len(S) else np.empty(0, np.uint64)
        got = i.cpu().numpy().astype(np.uint64) * np.uint64(max(len(S), 1)) + j.cpu().numpy().astype(np.uint64)
        assert_same(got, want, f"fp32 stage join {k}")


def test_batched_screen_error_within_certified_radius():
    """The sampled screen error of a batched pass (several dimension classes) stays inside the
    certified radius, and the diagnostic pass changes no pair."""
    joins = _ragged(16, 44)
    dev = [(torch.from_numpy(R).cuda(), torch.from_numpy(S).cuda(), float(np.sqrt(T))) for R, S, T in joins]
    for screen in ("bf16", "bf16x3"):
        res = tj.join_batched_result(dev, screen=screen, screen_diag=True)
        st = res.stats
        assert st["screen_err_pairs"] > 0
        assert st["screen_err_over_bound"] < 1.0, st
        plain = tj.join_batched_result(dev, screen=screen)
        assert torch.equal(res.keys(), plain.keys())


@pytest.mark.parametrize("four", [False, True])
def test_int14_many_items_exact(four):
    """Many tile pairs per CTA (30,000 rows, d = 128): the four-product screen's on-demand x / ll
    products and their hand-off between the epilogue warps and the UMMA issuer, and the high-limb
    screen's resident R tiles over whole chunks and its four accumulators, give the oracle's pairs."""
    w = W.int14x128(n=30000, samples=1 << 14)
    k, st = gpu_keys(w.R, None, w.T, "upper", "int8limb", i8_four_products=four)
    assert_same(k, oracle.join_i16(w.R, None, w.T, "upper"), "int14 n=30000")
    assert st["tile_pairs"] > 148 * 40
