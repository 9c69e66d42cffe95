"""Autotuner over the join's tile shapes and variants, keyed by (d, dtype, screen, mode, size, selectivity).

What it chooses, per workload (every choice gives the same pair set; only the time differs):

* ``screen``       -- the screen's operand format when the caller asks for ``screen="auto"``:
                      BF16 or FP16, single or hi/lo-split (x3) operands;
* ``cta_pair``     -- BM x BN: 256 x 256 tiles on a CTA pair (cta_group::2) or 128 x 256 on one SM;
* ``half_pack``    -- one SM: 128 x 128 half-items with dead halves dropped, or whole 128 x 256 items;
* ``k_block``      -- BK: elements of K per pipeline stage (64, 32 or 16);
* ``stages``       -- operand stages in flight (2 up to the compiled count);
* ``i8_four_products`` -- limb count of the int14 screen: the high-limb product only (undecided
                      pairs refined exactly) or all four limb products decided in the kernel;
* ``chunk_items``  -- tile pairs per chunk of the persistent screen's work queue;
* ``index_frame``  -- cells over input dimensions or over principal directions;
* ``band_fp32``    -- the certified FP32 band stage in front of the FP64 terminal.

The space is searched coordinate by coordinate in the order above: each dimension's values are
timed with the others held at the best so far (the library's own device time of the whole join,
best of ``reps``, on an evenly spaced row sample of the caller's data), so a tuning costs about
twenty sample joins instead of the product of all options.  Every timed choice must give the same
pair count.  The result is stored under a key of d, dtype, requested screen, mode, the log2 size
of the pair space and the log2 selectivity (result pairs per row); tables persist as JSON.

``default_table()`` is the table committed with the package (``tuned_b200.json``, produced by
``python -m tensorjoin_variants_b200.autotune`` on a B200 over the five benchmark configurations);
``api.join(..., screen="auto")`` and ``Tuner.join`` consult it before tuning.

The reference has no autotuner (its kernels state "no autotuned configurations",
tensorjoin_20260902_certified_exact_join/two_gate_campaign_20260908/src/g2_kernels.py:1).
"""
from __future__ import annotations

import json
import math
import os
import threading
from dataclasses import asdict, dataclass, replace
from pathlib import Path
from typing import Callable

import torch

from . import api
from ._lib import TJError

DEFAULT_TABLE = Path(__file__).resolve().parent / "tuned_b200.json"
FLOAT_SCREENS = ("bf16x3", "fp16x3", "bf16", "fp16")


@dataclass(frozen=True)
class Choice:
    screen: str = ""              # "": the screen the caller asked for
    cta_pair: bool = True
    half_pack: bool = True        # one-SM screen: dead 128-row halves of candidate tile pairs dropped
    k_block: int = 0              # 0: by d (64 for rows of more than 32 elements)
    stages: int = 0               # 0: every compiled stage
    i8_four_products: bool = False
    chunk_items: int = 0          # 0: the library default (64)
    index_frame: str = "auto"
    band_fp32: bool = False

    def kwargs(self) -> dict:
        kw = dict(cta_pair=self.cta_pair, chunk_items=self.chunk_items, index_frame=self.index_frame,
                  band_fp32=self.band_fp32, k_block=self.k_block, stages=self.stages,
                  i8_four_products=self.i8_four_products, half_pack=self.half_pack)
        return kw

    def screen_for(self, requested: str) -> str:
        return self.screen or requested


CHUNK_ITEMS = (16, 64, 256)


def dimensions(d: int, screen: str, mode: str) -> list[tuple[str, list]]:
    """Per dimension, the values that change what runs for this (d, requested screen, mode); the
    first value of each list is the library's default."""
    kpad = 16 if d <= 16 else 32 if d <= 32 else 64 * ((d + 63) // 64)
    dims: list[tuple[str, list]] = []
    if screen == "auto":
        dims.append(("screen", list(FLOAT_SCREENS)))
    float_screen = screen != "int8limb" and screen != "plain"
    if float_screen and mode == "rs" and d >= 256:
        dims.append(("cta_pair", [True, False]))
    if float_screen:
        dims.append(("half_pack", [True, False]))
    if screen == "int8limb" and kpad <= 256:
        dims.append(("i8_four_products", [False, True]))
    if float_screen:
        kbs = [0] + [k for k in (32, 16) if k < min(kpad, 64) and kpad % k == 0]
        if len(kbs) > 1:
            dims.append(("k_block", kbs))
        dims.append(("stages", [0, 3, 2]))
    dims.append(("chunk_items", [0] + [c for c in CHUNK_ITEMS if c != 64]))
    if 9 <= d <= 128:
        dims.append(("index_frame", ["axes", "pca"]))
    if float_screen:
        dims.append(("band_fp32", [False, True]))
    return dims


def candidates(d: int, screen: str, mode: str) -> list[Choice]:
    """Every single-coordinate variation of the default choice (the first sweep of the search)."""
    out = [Choice()]
    for name, values in dimensions(d, screen, mode):
        for v in values[1:]:
            out.append(replace(Choice(), **{name: v}))
    return out


def tune_key(d: int, dtype: str, screen: str, mode: str, n_rows: int, n_cols: int, per_row: float) -> str:
    """Table key: the log2 of the pair space and of the result pairs per row, rounded."""
    space = max(1, n_rows) * max(1, n_cols)
    return (f"d{d}/{dtype}/{screen}/{mode}/space2^{int(round(math.log2(space)))}"
            f"/sel2^{int(round(math.log2(1.0 + max(0.0, per_row))))}")


def _sample_rows(X: torch.Tensor, k: int) -> torch.Tensor:
    """An evenly spaced sample of k rows (all rows when k <= 0 or k >= n)."""
    n = X.shape[0]
    if k <= 0 or n <= k:
        return X
    idx = torch.linspace(0, n - 1, k, device=X.device).round().long()
    return X.index_select(0, idx).contiguous()


_DEFAULT = None


def default_table() -> "Tuner":
    """The committed B200 table (read-only use; empty if the file is absent)."""
    global _DEFAULT
    if _DEFAULT is None:
        _DEFAULT = Tuner(str(DEFAULT_TABLE) if DEFAULT_TABLE.exists() else None, read_only=True)
    return _DEFAULT


class Tuner:
    """Per-key table of the fastest ``Choice``; thread-safe; optional JSON persistence."""

    def __init__(self, path: str | None = None, read_only: bool = False):
        self.path = path
        self.read_only = read_only
        self.table: dict[str, dict] = {}
        self._lock = threading.Lock()
        if path and os.path.exists(path):
            with open(path) as f:
                self.table = json.load(f)

    # ---------------------------------------------------------------- table
    def lookup(self, key: str) -> Choice | None:
        with self._lock:
            e = self.table.get(key)
        return Choice(**e["choice"]) if e else None

    def record(self, key: str, best: Choice, timings: dict[str, float]) -> None:
        with self._lock:
            self.table[key] = {"choice": asdict(best), "ms": timings}
            if self.path and not self.read_only:
                tmp = self.path + ".tmp"
                with open(tmp, "w") as f:
                    json.dump(self.table, f, indent=1, sort_keys=True)
                os.replace(tmp, self.path)

    # ---------------------------------------------------------------- measuring
    @staticmethod
    def pick(cands: list[Choice], runner: Callable[[Choice], tuple[float, int]], reps: int = 2,
             count: int | None = None):
        """Run every candidate ``reps`` times through ``runner`` (-> (ms, result pairs), or None when
        the choice cannot run on this data); the fastest by its best time wins, ties to the earlier
        candidate.  Returns (best, timings, result pairs)."""
        timings: dict[str, float] = {}
        best, best_ms = None, math.inf
        for c in cands:
            ms = math.inf
            for _ in range(max(1, reps)):
                r = runner(c)
                if r is None:
                    break
                t, n = r
                if count is None:
                    count = n
                elif n != count:
                    raise RuntimeError(f"choice {c} changed the pair count ({n} != {count})")
                ms = min(ms, t)
            timings[json.dumps(asdict(c), sort_keys=True)] = ms
            if ms < best_ms:
                best, best_ms = c, ms
        if best is None:
            raise RuntimeError("no candidate could run")
        return best, timings, count or 0

    @classmethod
    def search(cls, d: int, screen: str, mode: str, runner: Callable[[Choice], tuple[float, int] | None],
               reps: int = 2):
        """Coordinate search: each dimension's values timed with the others at the best so far."""
        best = Choice()
        timings: dict[str, float] = {}
        count = None
        for name, values in dimensions(d, screen, mode):
            cands = [replace(best, **{name: v}) for v in values]
            best, t, count = cls.pick(cands, runner, reps, count)
            timings.update(t)
        return best, timings, count or 0

    @staticmethod
    def _device_runner(R, S, eps2, mode, screen):
        def run(c: Choice):
            try:
                res = api.join_result(R, S, eps2=eps2, mode=mode, screen=c.screen_for(screen), **c.kwargs())
            except TJError as e:
                if e.code in (-4, -7):   # FP16 range exceeded / combination not supported: skip
                    return None
                raise
            st = res.stats
            return float(st["ms_total"]), int(st["result_pairs"])
        return run

    def _sample(self, R, S, mode, sample_rows):
        """Row sample for tuning: R rows against all of S (R-S), or a sample self-join, with the
        factor that scales its result pairs per row to the full join."""
        if mode == "rs":
            Rs = _sample_rows(R, sample_rows)
            return Rs, S, 1.0
        Xs = _sample_rows(R, sample_rows)
        return Xs, None, R.shape[0] / max(1, Xs.shape[0])

    def tune(self, R, S, eps2: float, mode: str = "rs", screen: str = "bf16", sample_rows: int = 4096,
             reps: int = 2) -> tuple[Choice, str, dict]:
        """Search the choices on a row sample and record the fastest; returns (choice, key, timings)."""
        Rt, _ = api._as_device(R, screen == "int8limb")
        St = None if S is None else api._as_device(S, screen == "int8limb")[0]
        Rs, Ss, scale = self._sample(Rt, St, mode, sample_rows)
        d = Rt.shape[1]
        best, timings, count = self.search(d, screen, mode, self._device_runner(Rs, Ss, eps2, mode, screen), reps)
        per_row = count / max(1, Rs.shape[0]) * scale
        key = tune_key(d, _dtype(Rt), screen, mode, Rt.shape[0], Rt.shape[0] if St is None else St.shape[0], per_row)
        self.record(key, best, timings)
        return best, key, timings

    def key_for(self, R, S, eps2: float, mode: str, screen: str, probe_rows: int = 512) -> str:
        """Key of the full join, with the selectivity measured on a small row sample."""
        Rt, _ = api._as_device(R, screen == "int8limb")
        St = None if S is None else api._as_device(S, screen == "int8limb")[0]
        Rs, Ss, scale = self._sample(Rt, St, mode, probe_rows)
        probe = "bf16x3" if screen == "auto" else screen
        res = api.join_result(Rs, Ss, eps2=eps2, mode=mode, screen=probe)
        per_row = res.count / max(1, Rs.shape[0]) * scale
        return tune_key(Rt.shape[1], _dtype(Rt), screen, mode, Rt.shape[0],
                        Rt.shape[0] if St is None else St.shape[0], per_row)

    def choose(self, R, S, eps2: float, mode: str, screen: str, sample_rows: int = 4096,
               tune_on_miss: bool = True) -> tuple[Choice, str]:
        """The choice for this join: this table, then the committed default table, then (on a miss)
        a tuning run on a sample, or the library defaults when tuning is off."""
        key = self.key_for(R, S, eps2, mode, screen)
        choice = self.lookup(key)
        if choice is None and self is not default_table():
            choice = default_table().lookup(key)
        if choice is None:
            if not tune_on_miss:
                return Choice(screen="bf16x3" if screen == "auto" else ""), key
            # the tuning sample may bucket its selectivity differently: keep both keys
            choice, _, timings = self.tune(R, S, eps2, mode, screen, sample_rows)
            self.record(key, choice, timings)
        return choice, key

    def join(self, R, S=None, eps=None, *, eps2=None, mode: str = "rs", screen: str = "bf16",
             sample_rows: int = 4096) -> api.Result:
        """Run the join with the table's choice for its key, tuning first on a miss."""
        T = api._threshold(eps, eps2)
        choice, _ = self.choose(R, S, T, mode, screen, sample_rows)
        return api.join_result(R, S, eps2=T, mode=mode, screen=choice.screen_for(screen), **choice.kwargs())

    # ---------------------------------------------------------------- batched joins
    @staticmethod
    def batch_key(joins, screen: str) -> str:
        """Key of a batch: the dimensions present, the requested screen, the number of joins and the
        log2 of the batch's pair space."""
        dims = sorted({int(j[0].shape[1]) for j in joins})
        space = sum(int(j[0].shape[0]) * int(j[1].shape[0]) for j in joins)
        return (f"batch/d{'-'.join(map(str, dims))}/f32/{screen}/joins2^{int(round(math.log2(max(1, len(joins)))))}"
                f"/space2^{int(round(math.log2(max(1, space))))}")

    def batch_choice(self, joins, screen: str):
        """This table's (then the committed table's) choice for the batch, or None; no tuning."""
        key = self.batch_key(joins, screen)
        return self.lookup(key) or default_table().lookup(key)

    def join_batched(self, joins, screen: str = "bf16x3", sample_joins: int = 64, reps: int = 2,
                     fresh: bool = False):
        """Tuned batched join: the choice is searched on a seeded sample of the batch's joins (the
        batch's own mix of sizes and dimensions), keyed as ``batch_key``; ``fresh`` searches even
        when a table already holds the key."""
        dims = sorted({int(j[0].shape[1]) for j in joins})
        key = self.batch_key(joins, screen)
        choice = None if fresh else (self.lookup(key) or default_table().lookup(key))
        if choice is None:
            g = torch.Generator().manual_seed(len(joins))
            idx = torch.randperm(len(joins), generator=g)[:sample_joins].tolist()
            sample = [joins[i] for i in sorted(idx)]

            def run(c: Choice):
                kw = c.kwargs()
                kw.pop("i8_four_products")
                try:
                    res = api.join_batched_result(sample, screen=c.screen_for(screen), **kw)
                except TJError as e:
                    if e.code in (-4, -7):
                        return None
                    raise
                return float(res.stats["ms_total"]), int(res.stats["result_pairs"])

            best, timings, _ = self.search(max(dims), screen, "rs", run, reps)
            self.record(key, best, timings)
            choice = best
        kw = choice.kwargs()
        kw.pop("i8_four_products")
        return api.join_batched_result(joins, screen=choice.screen_for(screen), **kw), choice


def _dtype(t: torch.Tensor) -> str:
    return "i16" if t.dtype == torch.int16 else "f32"


def _produce(path: str, sample_rows: int) -> None:
    """Tune the five benchmark configurations (seeded synthetic data of their shapes) on this GPU
    and write the table to `path`; sample_rows <= 0 times every choice on the full configuration (the
    batch on all of its joins), which is what the benchmark runs: choices timed on a row sample
    did not carry over to the full joins, whose tile-pair density and pruning differ."""
    from . import workloads as W

    t = Tuner(path)
    jobs = [("factor512", "fp16", "rs"), ("factor512", "auto", "rs"), ("mixture64", "bf16x3", "rs"),
            ("mixture64", "auto", "rs"), ("int14x128", "int8limb", "upper"), ("uniform16", "plain", "upper")]
    for name, screen, mode in jobs:
        w = getattr(W, name)()
        R = torch.from_numpy(w.R).cuda()
        S = None if w.S is None else torch.from_numpy(w.S).cuda()
        key = t.key_for(R, S, float(w.T), mode, screen)
        choice, _, timings = t.tune(R, S, float(w.T), mode, screen, sample_rows)   # always searched afresh
        t.record(key, choice, timings)
        print(f"{name} {screen}: {key} -> {choice}", flush=True)
        del R, S
    joins, classes = W.ragged4096_device()
    _, choice = t.join_batched(joins, "bf16x3", sample_joins=len(joins) if sample_rows <= 0 else 64, fresh=True)
    print(f"ragged4096 bf16x3: {t.batch_key(joins, 'bf16x3')} -> {choice}", flush=True)
    del joins, classes
    print(json.dumps(t.table, indent=1, sort_keys=True))


if __name__ == "__main__":
    import argparse

    ap = argparse.ArgumentParser(description="tune the benchmark configurations and write a table")
    ap.add_argument("--out", default=str(DEFAULT_TABLE))
    ap.add_argument("--sample-rows", type=int, default=0, help="rows per tuning sample (0: the full configuration)")
    a = ap.parse_args()
    _produce(a.out, a.sample_rows)


__all__ = ["Choice", "Tuner", "candidates", "dimensions", "tune_key", "default_table", "CHUNK_ITEMS"]
