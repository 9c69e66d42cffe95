"""GPU tests of each stage on its own, against the CPU oracle, and of the bounded-wait path.

* Per-stage audit: the screen's certified accepts must all be oracle pairs (no false accept), every
  oracle pair must be a certified accept or in the band (no false reject), and the refinement must
  accept exactly the band's oracle pairs.  The reference audited each stage of its cascade the same
  way and froze the expected counts (tensorjoin_20260902_certified_exact_join/src/run_g2a_tensorjoin.py:384-469,
  src/run_g4a_dynamic_router_timing.py:56-61); here every expected false count is zero.
* Timeout path: with the pipeline wait limit set to 1 us through the C ABI, every screen kernel gives
  up inside its first waits, drains its own copies and tensor-core work, frees its tensor memory and
  the join fails with TJ_ERR_TIMEOUT; the same join at the default limit then matches the oracle
  (the context is still usable).  No fault, trap or hang is involved: the waits are ordinary bounded
  waits that run out.
* Neighbour table: GDS-Join's counts-plus-flat-list output (adapters/gds_g2a/main.cu:488-540) against
  a table built from the oracle's pairs on GDS's own 2-D test set.
"""
import ctypes as C
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


def _join(R, S, T, mode, screen, **kw):
    Rt = torch.from_numpy(np.ascontiguousarray(R)).cuda()
    St = None if S is None else torch.from_numpy(np.ascontiguousarray(S)).cuda()
    return tj.join_result(Rt, St, eps2=T, mode=mode, screen=screen, guards=True, **kw)


def _np(t):
    return t.cpu().numpy().view(np.uint64)


def _to_upper(keys, n):
    """Directed/upper oracle keys -> the screen's i < j form (self-joins)."""
    i, j = keys // np.uint64(n), keys % np.uint64(n)
    keep = i < j
    return np.sort(i[keep] * np.uint64(n) + j[keep])


def _cases():
    mix = W.mixture64(n=6000, samples=1 << 16)
    uni = W.uniform16(n=5000)
    fac = W.factor512(n=2048, samples=1 << 15)
    i14 = W.int14x128(n=6000, samples=1 << 14)
    rng = np.random.default_rng(2000 + 1500 + 512)   # every tile pair a candidate: the CTA-pair screen runs
    gR = (rng.standard_normal((2000, 512)) / np.sqrt(512)).astype(np.float32)
    gS = (rng.standard_normal((1500, 512)) / np.sqrt(512)).astype(np.float32)
    gT = float(np.quantile(((gR[:60, None, :].astype(np.float64) - gS[None, :300, :]) ** 2).sum(-1), 0.01))
    return {"mixture64": (mix.R, mix.S, mix.T, "rs"), "uniform16": (uni.R, None, uni.T, "upper"),
            "factor512": (fac.R, fac.S, fac.T, "rs"), "int14x128": (i14.R, None, i14.T, "upper"),
            "gauss512": (gR, gS, gT, "rs")}


_CASES = {}


def case(name):
    if not _CASES:
        _CASES.update(_cases())
    return _CASES[name]


STAGE_RUNS = [("mixture64", s, {}) for s in ("plain", "bf16", "fp16", "bf16x3", "fp16x3")] + \
             [("uniform16", s, {}) for s in ("plain", "bf16", "bf16x3")] + \
             [("factor512", "fp16", {}), ("factor512", "bf16", {}), ("factor512", "fp16", {"cta_pair": False}),
              ("gauss512", "fp16", {}),
              ("mixture64", "bf16x3", {"band_fp32": True}),
              ("int14x128", "int8limb", {}), ("int14x128", "int8limb", {"i8_four_products": True})]


@pytest.mark.parametrize("name,screen,kw", STAGE_RUNS,
                         ids=[f"{n}-{s}-{'-'.join(k) or 'default'}" for n, s, k in STAGE_RUNS])
def test_stage_audit(name, screen, kw):
    R, S, T, mode = case(name)
    n_cols = (R if S is None else S).shape[0]
    want = oracle.join_i16(R, S, T, mode) if R.dtype == np.int16 else oracle.join_f32(R, S, T, mode)
    res = _join(R, S, T, mode, screen, stage_keys=True, **kw)
    st = res.stats
    acc0 = _np(res.stage_keys(0))
    band = _np(res.stage_keys(1))
    assert len(acc0) == st["screen_accept"] and len(band) == st["band"]
    want_u = want if mode == "rs" else _to_upper(want, n_cols)
    false_accept = np.setdiff1d(acc0, want_u)
    false_reject = np.setdiff1d(want_u, np.union1d(acc0, band))
    assert false_accept.size == 0, f"screen accepted {false_accept.size} pairs the oracle rejects"
    assert false_reject.size == 0, f"screen rejected {false_reject.size} oracle pairs"
    assert np.intersect1d(acc0, band).size == 0
    band_in = np.intersect1d(band, want_u)
    assert band_in.size == st["refine_accept"], (band_in.size, st["refine_accept"])
    assert np.array_equal(_np(res.keys()), want)
    if screen == "int8limb" and kw.get("i8_four_products"):
        assert len(band) == 0


# ---------------------------------------------------------------- bounded waits
TIMEOUT_RUNS = [("mixture64", "bf16", {}), ("mixture64", "bf16x3", {}), ("gauss512", "fp16", {}),
                ("gauss512", "fp16", {"cta_pair": False}), ("int14x128", "int8limb", {}),
                ("int14x128", "int8limb", {"i8_four_products": True}), ("uniform16", "plain", {})]


@pytest.fixture
def wait_limit():
    L = _lib.lib()
    yield lambda ns: _lib.check(L.tj_set_wait_limit(int(ns)))
    _lib.check(L.tj_set_wait_limit(0))


@pytest.mark.parametrize("name,screen,kw", TIMEOUT_RUNS,
                         ids=[f"{n}-{s}-{'-'.join(k) or 'default'}" for n, s, k in TIMEOUT_RUNS])
def test_pipeline_wait_timeout_then_recovery(name, screen, kw, wait_limit):
    R, S, T, mode = case(name)
    want = oracle.join_i16(R, S, T, mode) if R.dtype == np.int16 else oracle.join_f32(R, S, T, mode)
    wait_limit(1000)   # 1 us: shorter than a tile's first copy and MMA
    if screen == "plain":   # the plain screen has no pipeline waits: the limit changes nothing
        assert np.array_equal(_np(_join(R, S, T, mode, screen, **kw).keys()), want)
    else:
        with pytest.raises(_lib.TJError) as e:
            _join(R, S, T, mode, screen, **kw)
        assert e.value.code == -5, e.value
    wait_limit(0)
    res = _join(R, S, T, mode, screen, **kw)
    if name == "gauss512":
        assert res.stats["screen_pair"] == (1 if kw.get("cta_pair", True) else 0)
    assert np.array_equal(_np(res.keys()), want)


def test_wait_limit_rejects_negative():
    assert _lib.lib().tj_set_wait_limit(-1) == -1
    _lib.check(_lib.lib().tj_set_wait_limit(0))


def test_batched_timeout_then_recovery(wait_limit):
    rng = np.random.default_rng(77)
    joins = []
    for k in range(24):
        d = (8, 32, 128)[k % 3]
        c = rng.random((8, d))
        R = (c[rng.integers(0, 8, 900)] + rng.standard_normal((900, d)) * 0.05).astype(np.float32)
        S = (c[rng.integers(0, 8, 1100)] + rng.standard_normal((1100, d)) * 0.05).astype(np.float32)
        joins.append((R, S, W.ragged_eps2(1100, d, 8, 0.05, 16)))
    dev = [(torch.from_numpy(R).cuda(), torch.from_numpy(S).cuda(), float(np.sqrt(T))) for R, S, T in joins]
    wait_limit(1000)
    with pytest.raises(_lib.TJError) as e:
        tj.join_batched(dev, screen="bf16x3")
    assert e.value.code == -5
    wait_limit(0)
    out = tj.join_batched(dev, screen="bf16x3")
    for (R, S, T), (i, j), (_, _, e) in zip(joins, out, dev):
        got = i.cpu().numpy().astype(np.uint64) * np.uint64(S.shape[0]) + j.cpu().numpy().astype(np.uint64)
        assert np.array_equal(got, oracle.join_f32(R, S, e * e, "rs"))


# ---------------------------------------------------------------- neighbour table
@pytest.mark.parametrize("screen", ["plain", "bf16x3"])
def test_neighbor_table_against_oracle(screen):
    """GDS's 100,000-point 2-D test set at eps = 1.0: per-row neighbour counts and the flat,
    row-ordered neighbour lists (self included, GDS's convention) equal a table built from the oracle."""
    X = np.load(GOLDEN / "gds_test_dat_f32.npy")
    n = len(X)
    want = oracle.join_f32(X, None, 1.0, "directed")
    wi, wj = oracle.keys_to_ij(want, n)
    want_counts = np.bincount(wi, minlength=n)
    res = _join(X, None, 1.0, "directed", screen)
    counts, flat = res.neighbor_table()
    assert np.array_equal(counts.cpu().numpy().astype(np.int64), want_counts)
    assert np.array_equal(flat.cpu().numpy(), wj)
    assert int(want_counts.sum()) == 27_982_024   # the FP64 oracle's count (GDS's FP32 run: 27,982,028)


# ---------------------------------------------------------------- the accumulation premise in isolation
def _premise_rows(rng, n, form, d=512, L=128.0):
    """Rows whose every entry is exact in BF16 and in FP16 (at most 8 significant bits, exponents in
    [-8, 7]), built so that the tensor-core sum of a pair runs through large partial sums while
    small products arrive: form 'x' and 'y' of four families, n // 4 rows each."""
    s = 243.0 / 8192.0                      # s * s = 0.45 ulp of L^2 in FP32: lost by a rounded sum
    out = np.zeros((n, d), np.float64)
    q = n // 4
    for f in range(4):
        for r in range(f * q, (f + 1) * q):
            # small entries of one sign: their products all add up (none cancel), the worst case for
            # products lost against a large running sum
            v = s * rng.choice([1.0, 0.5], d)
            if f == 0:     # +L^2 first, -L^2 last: every small product meets a running sum of ~L^2
                v[0] = L
                v[d - 1] = L if form == "x" else -L
            elif f == 1:   # the large pair cancels inside the first k-steps
                v[0] = L
                v[1] = L if form == "x" else -L
            elif f == 2:   # alternating large products in the first 64 k: the running sum oscillates
                for k in range(0, 64, 2):
                    v[k] = L if form == "x" else (L if (k // 2) % 2 == 0 else -L)
            else:          # random signs, magnitudes 2^-8 .. 2^7 with 6 significant bits
                e = rng.integers(-8, 8, d).astype(np.float64)
                m = rng.integers(32, 64, d).astype(np.float64) / 64.0
                v = rng.choice([-1.0, 1.0], d) * m * 2.0 ** e
            out[r] = v
    return out.astype(np.float32)


@pytest.mark.parametrize("screen", ["fp16", "bf16", "fp16x3", "bf16x3"])
def test_accumulation_premise(screen):
    """The certificate assumes every FP32 accumulation step of the tensor core errs by at most
    2 ulp of the running sum, |p - z.w| <= gamma ||z|| ||w|| + c0 with gamma = (K + 64) 2^-22.
    Rows are exact in the operand format and symmetric about 0 (R = [A; -A], S = [B; -B]), so the
    centre is exactly 0, the operand rows equal the input rows and every other term of the certified
    radius vanishes: the screen's diagnostic ratio |d2hat - d2| / radius is then
    |p - x.y| / (gamma ||z|| ||w|| + c0) up to the FP64 norm roundings (~1e-16 relative).  Every
    accumulator of the one tile pair (128 x 256) is dumped and compared."""
    rng = np.random.default_rng(99)
    A = _premise_rows(rng, 64, "x")
    B = _premise_rows(rng, 128, "y")
    R = np.concatenate([A, -A])
    S = np.concatenate([B, -B])
    T = float(np.median(oracle.pair_d2(R, S, np.arange(128), np.arange(128))))
    res = _join(R, S, T, "rs", screen, screen_diag=True)
    st = res.stats
    assert st["screen_err_pairs"] == 128 * 256, st
    ratio = st["screen_err_over_bound"]
    print(f"premise {screen}: max |p - x.y| / (gamma |z||w| + c0) = {ratio:.4f}, "
          f"max |d2hat - d2| = {st['screen_max_abs_err']:.3e}")
    assert ratio < 1.0, st
    assert np.array_equal(_np(res.keys()), oracle.join_f32(R, S, T, "rs"))


# ---------------------------------------------------------------- half-tile packing and tile-shape knobs
@pytest.mark.parametrize("screen", ["bf16x3", "fp16", "bf16"])
def test_half_packing_same_pairs_fewer_evaluations(screen):
    """Dropping dead 128-row halves of candidate tile pairs (the default) gives the oracle's pairs with
    no more distance evaluations than screening whole tile pairs; the tile-shape knobs (k-block,
    stages) give the same pairs too."""
    R, S, T, mode = case("mixture64")
    want = oracle.join_f32(R, S, T, mode)
    packed = _join(R, S, T, mode, screen)
    whole = _join(R, S, T, mode, screen, half_pack=False)
    assert np.array_equal(_np(packed.keys()), want)
    assert np.array_equal(_np(whole.keys()), want)
    assert packed.stats["pairs_screened"] <= whole.stats["pairs_screened"]
    assert packed.stats["screen_ops_issued"] <= whole.stats["screen_ops_issued"]
    for kb, stg in ((32, 0), (16, 3), (0, 2)):
        r = _join(R, S, T, mode, screen, k_block=kb, stages=stg)
        assert np.array_equal(_np(r.keys()), want), (kb, stg)


def test_half_packing_self_join_and_batched():
    R, S, T, mode = case("uniform16")
    want = oracle.join_f32(R, None, T, "upper")
    for hp in (True, False):
        assert np.array_equal(_np(_join(R, None, T, "upper", "bf16x3", half_pack=hp).keys()), want)
    rng = np.random.default_rng(78)
    joins = []
    for k in range(20):
        d = (8, 32, 128)[k % 3]
        c = rng.random((8, d))
        Rk = (c[rng.integers(0, 8, 700)] + rng.standard_normal((700, d)) * 0.05).astype(np.float32)
        Sk = (c[rng.integers(0, 8, 1900)] + rng.standard_normal((1900, d)) * 0.05).astype(np.float32)
        joins.append((Rk, Sk, W.ragged_eps2(1900, d, 8, 0.05, 16)))
    dev = [(torch.from_numpy(a).cuda(), torch.from_numpy(b).cuda(), float(np.sqrt(t))) for a, b, t in joins]
    for hp in (True, False):
        out = tj.join_batched(dev, screen="bf16x3", half_pack=hp, guards=True)
        for (Rk, Sk, t), (i, j), (_, _, e) in zip(joins, out, dev):
            got = i.cpu().numpy().astype(np.uint64) * np.uint64(Sk.shape[0]) + j.cpu().numpy().astype(np.uint64)
            assert np.array_equal(got, oracle.join_f32(Rk, Sk, e * e, "rs"))
