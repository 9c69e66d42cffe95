"""Autotuner host logic on the CPU (selection, keys, persistence) and, on a GPU, tuned joins
that give the oracle's pairs and reuse the table."""
import json

import numpy as np
import pytest

from tensorjoin_variants_b200 import autotune as A


def test_dimensions_cover_only_what_applies():
    d512 = dict(A.dimensions(512, "fp16", "rs"))
    assert d512["cta_pair"] == [True, False]                    # BM x BN: CTA pair or one SM
    assert d512["k_block"] == [0, 32, 16] and d512["stages"] == [0, 3, 2]
    assert "index_frame" not in d512                            # d > 128: no principal-direction cells
    assert d512["band_fp32"] == [False, True]
    assert set(d512["chunk_items"]) == {0, 16, 256}
    d64 = dict(A.dimensions(64, "bf16x3", "upper"))
    assert "cta_pair" not in d64                                # self-join / d < 256: one-SM screen only
    assert d64["index_frame"] == ["axes", "pca"]
    d8 = dict(A.dimensions(8, "bf16", "rs"))
    assert "k_block" not in d8                                  # a 16-element row has one k-block size
    di = dict(A.dimensions(128, "int8limb", "upper"))
    assert di["i8_four_products"] == [False, True]              # limb count of the int14 screen
    assert "band_fp32" not in di and "k_block" not in di
    assert "i8_four_products" not in dict(A.dimensions(300, "int8limb", "upper"))   # rows > 256: four products
    da = dict(A.dimensions(64, "auto", "rs"))
    assert da["screen"] == list(A.FLOAT_SCREENS)                # operand format chosen by the tuner
    c = A.candidates(64, "bf16x3", "rs")
    assert c[0] == A.Choice() and len(set(c)) == len(c)


def test_coordinate_search_keeps_each_dimensions_best():
    """Each dimension's best is kept while the next one is searched; interactions add up."""
    def runner(ch):
        ms = 10.0 - (2.0 if ch.chunk_items == 256 else 0.0) - (1.5 if ch.index_frame == "pca" else 0.0)
        ms -= 0.5 if ch.stages == 3 else 0.0
        return ms, 77
    best, timings, count = A.Tuner.search(64, "bf16x3", "rs", runner, reps=1)
    assert (best.chunk_items, best.index_frame, best.stages) == (256, "pca", 3)
    assert count == 77 and min(timings.values()) == 6.0


def test_search_skips_choices_that_cannot_run():
    def runner(ch):
        if ch.screen.startswith("fp16"):
            return None                                         # e.g. FP16 range exceeded
        return (1.0 if ch.screen == "bf16" else 2.0), 5
    best, _, _ = A.Tuner.search(64, "auto", "rs", runner, reps=1)
    assert best.screen == "bf16"


def test_tune_key_buckets():
    k = A.tune_key(64, "f32", "bf16x3", "rs", 1 << 20, 1 << 20, 15.0)
    assert k == "d64/f32/bf16x3/rs/space2^40/sel2^4"
    assert A.tune_key(64, "f32", "bf16x3", "rs", 1 << 20, 1 << 20, 16.5) == k   # same bucket
    assert A.tune_key(64, "f32", "bf16x3", "rs", 1 << 20, 1 << 20, 0.0).endswith("sel2^0")
    assert A.tune_key(64, "f32", "bf16x3", "rs", 1 << 21, 1 << 20, 15.0) != k


def test_pick_fastest_by_best_time_and_ties_to_first():
    cands = [A.Choice(chunk_items=c) for c in (16, 64, 256)]
    times = {16: [5.0, 4.0], 64: [3.0, 3.5], 256: [3.0, 9.0]}
    calls = {c: 0 for c in (16, 64, 256)}

    def runner(ch):
        k = ch.chunk_items
        t = times[k][calls[k]]
        calls[k] += 1
        return t, 1234

    best, timings, count = A.Tuner.pick(cands, runner, reps=2)
    assert best.chunk_items == 64 and count == 1234
    assert len(timings) == 3 and min(timings.values()) == 3.0
    assert all(v == 2 for v in calls.values())


def test_pick_rejects_a_choice_that_changes_the_pairs():
    cands = [A.Choice(chunk_items=16), A.Choice(chunk_items=64)]
    with pytest.raises(RuntimeError):
        A.Tuner.pick(cands, lambda ch: (1.0, 10 if ch.chunk_items == 16 else 11), reps=1)


def test_table_persists(tmp_path):
    path = str(tmp_path / "tune.json")
    t = A.Tuner(path)
    choice = A.Choice(screen="fp16", cta_pair=False, k_block=32, stages=3, chunk_items=256, index_frame="pca",
                      band_fp32=True)
    t.record("d64/f32/bf16/rs/space2^30/sel2^3", choice, {"x": 1.5})
    again = A.Tuner(path)
    assert again.lookup("d64/f32/bf16/rs/space2^30/sel2^3") == choice
    assert again.lookup("missing") is None
    assert json.load(open(path))["d64/f32/bf16/rs/space2^30/sel2^3"]["ms"] == {"x": 1.5}


def test_batch_key_and_lookup(tmp_path):
    """A batch is keyed by its dimensions, screen, join count and pair space; the lookup returns the
    recorded choice without tuning."""
    joins = [(np.zeros((300, 8), np.float32), np.zeros((500, 8), np.float32), 0.1),
             (np.zeros((1000, 32), np.float32), np.zeros((40, 32), np.float32), 0.2)]
    key = A.Tuner.batch_key(joins, "bf16x3")
    assert key == "batch/d8-32/f32/bf16x3/joins2^1/space2^18"   # 190,000 pairs
    t = A.Tuner(str(tmp_path / "tune.json"))
    assert t.batch_choice(joins, "bf16x3") is None
    t.record(key, A.Choice(half_pack=False, stages=3), {})
    assert t.batch_choice(joins, "bf16x3") == A.Choice(half_pack=False, stages=3)
    assert t.batch_choice(joins, "fp16") is None


@pytest.mark.gpu
def test_tuned_join_matches_oracle_and_reuses_the_table(tmp_path):
    import torch

    import oracle
    from tensorjoin_variants_b200 import workloads as W

    w = W.mixture64(n=9000, samples=1 << 14)
    R, S = torch.from_numpy(w.R).cuda(), torch.from_numpy(w.S).cuda()
    tuner = A.Tuner(str(tmp_path / "t.json"))
    n_tunes = []
    orig = tuner.tune

    def counting_tune(*a, **k):
        n_tunes.append(1)
        return orig(*a, **k)

    tuner.tune = counting_tune
    want = oracle.join_f32(w.R, w.S, w.T, "rs")
    for _ in range(2):
        res = tuner.join(R, S, eps2=w.T, screen="bf16x3", sample_rows=2048)
        got = res.keys().cpu().numpy().view(np.uint64)
        assert np.array_equal(got, want)
    assert len(n_tunes) == 1                       # the second join found its key in the table
    X = torch.from_numpy(w.R[:4000]).cuda()
    res = tuner.join(X, None, eps2=w.T, mode="upper", screen="fp16", sample_rows=1024)
    assert np.array_equal(res.keys().cpu().numpy().view(np.uint64), oracle.join_f32(w.R[:4000], None, w.T, "upper"))


def test_tuner_join_flow_with_a_fake_library(monkeypatch, tmp_path):
    """Host flow of Tuner.join on the CPU: the selectivity probe, tuning on a miss (every candidate
    timed, the fastest kept under both the probe's and the tuning sample's keys), reuse on a hit,
    and the final join run with the chosen options."""
    import torch

    calls = []

    class FakeResult:
        def __init__(self, R, S, kw):
            rows = R.shape[0]
            self.count = rows * 12                                   # 12 result pairs per row
            ms = 9.0 - (2.0 if kw.get("chunk_items") == 256 else 0.0) - (2.0 if kw.get("index_frame") == "pca" else 0.0)
            self.stats = {"ms_total": ms, "result_pairs": self.count}

    def fake_join_result(R, S, eps2=None, mode="rs", screen="bf16", **kw):
        calls.append((R.shape[0], kw))
        return FakeResult(R, S, kw)

    monkeypatch.setattr(A.api, "join_result", fake_join_result)
    monkeypatch.setattr(A.api, "_as_device", lambda x, allow_int16: (x, False))
    R = torch.zeros((50000, 64))
    S = torch.zeros((60000, 64))
    tuner = A.Tuner(str(tmp_path / "t.json"))
    tuner.join(R, S, eps2=0.1, screen="bf16x3", sample_rows=1024)
    final_kw = calls[-1][1]
    assert calls[-1][0] == 50000 and final_kw["chunk_items"] == 256 and final_kw["index_frame"] == "pca"
    n_first = len(calls)
    n_search = sum(len(v) for _, v in A.dimensions(64, "bf16x3", "rs"))
    assert n_first == 1 + 2 * n_search + 1                                # probe, tuning (2 reps), join
    tuner.join(R, S, eps2=0.1, screen="bf16x3", sample_rows=1024)
    assert len(calls) == n_first + 2                                      # probe and join only
    key = A.tune_key(64, "f32", "bf16x3", "rs", 50000, 60000, 12.0)
    assert tuner.lookup(key) == A.Choice(chunk_items=256, index_frame="pca")
