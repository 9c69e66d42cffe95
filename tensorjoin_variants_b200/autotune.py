"""Autotuner for the join's run-time choices, keyed by (d, dtype, screen, mode, size, selectivity).

The kernels' tile shapes are fixed at compile time (128 x 256 items, or 256 x 256 on a CTA pair;
16-, 32- or 64-element k-blocks by d; stage counts by screen), so what is left to choose per
workload is which of those variants runs and how the work is cut:

* ``cta_pair``     -- the 2-SM (cta_group::2) screen or the one-SM screen, where both apply;
* ``chunk_items``  -- tile pairs per scheduling chunk of the persistent screen;
* ``index_frame``  -- cells over input dimensions or over principal directions;
* ``band_fp32``    -- the certified FP32 band stage in front of the FP64 terminal.

``Tuner.tune`` times every applicable combination on an evenly spaced row sample of the caller's
data (the library's own per-stage device times, best of ``reps``), keeps the fastest, and stores it
under a key built from d, dtype, screen, mode, the log2 size of the pair space and the log2
selectivity (result pairs per row) measured on the sample.  ``Tuner.join`` estimates the
selectivity on a small sample, looks the key up (tuning on a miss) and runs the full join with the
chosen options.  Every choice gives the same pair set; only the time differs.  The table can be
saved to and loaded from a JSON file.

The reference has no autotuner (its kernels state "no autotuned configurations",
tensorjoin_20260902_certified_exact_join/two_gate_campaign_20260908/src/g2_kernels.py:1).
"""
from __future__ import annotations

import itertools
import json
import math
import os
import threading
from dataclasses import asdict, dataclass
from typing import Callable

import torch

from . import api


@dataclass(frozen=True)
class Choice:
    cta_pair: bool = True
    chunk_items: int = 0          # 0: the library default (64)
    index_frame: str = "auto"
    band_fp32: bool = False

    def kwargs(self) -> dict:
        return dict(cta_pair=self.cta_pair, chunk_items=self.chunk_items, index_frame=self.index_frame,
                    band_fp32=self.band_fp32)


CHUNK_ITEMS = (16, 64, 256)


def candidates(d: int, screen: str, mode: str) -> list[Choice]:
    """Every combination whose options change what runs for this (d, screen, mode)."""
    pairs = [True, False] if (mode == "rs" and d >= 256 and screen in ("bf16", "fp16")) else [True]
    frames = ["axes", "pca"] if 9 <= d <= 128 else ["auto"]
    bands = [False, True] if screen in ("bf16", "fp16", "bf16x3", "fp16x3") else [False]
    return [Choice(p, c, f, b) for p, c, f, b in itertools.product(pairs, CHUNK_ITEMS, frames, bands)]


def tune_key(d: int, dtype: str, screen: str, mode: str, n_rows: int, n_cols: int, per_row: float) -> str:
    """Table key: the log2 of the pair space and of the result pairs per row, rounded."""
    space = max(1, n_rows) * max(1, n_cols)
    return (f"d{d}/{dtype}/{screen}/{mode}/space2^{int(round(math.log2(space)))}"
            f"/sel2^{int(round(math.log2(1.0 + max(0.0, per_row))))}")


def _sample_rows(X: torch.Tensor, k: int) -> torch.Tensor:
    n = X.shape[0]
    if n <= k:
        return X
    idx = torch.linspace(0, n - 1, k, device=X.device).round().long()
    return X.index_select(0, idx).contiguous()


class Tuner:
    """Per-key table of the fastest ``Choice``; thread-safe; optional JSON persistence."""

    def __init__(self, path: str | None = None):
        self.path = path
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
            if self.path:
                tmp = self.path + ".tmp"
                with open(tmp, "w") as f:
                    json.dump(self.table, f, indent=1, sort_keys=True)
                os.replace(tmp, self.path)

    # ---------------------------------------------------------------- measuring
    @staticmethod
    def pick(cands: list[Choice], runner: Callable[[Choice], tuple[float, int]], reps: int = 2):
        """Run every candidate ``reps`` times through ``runner`` (-> (ms, result pairs)); the
        fastest by its best time wins, ties to the earlier candidate.  Returns (best, timings,
        result pairs of the first run)."""
        timings: dict[str, float] = {}
        best, best_ms, count = None, math.inf, None
        for c in cands:
            ms = math.inf
            for _ in range(max(1, reps)):
                t, n = runner(c)
                if count is None:
                    count = n
                elif n != count:
                    raise RuntimeError(f"choice {c} changed the pair count ({n} != {count})")
                ms = min(ms, t)
            timings[json.dumps(asdict(c), sort_keys=True)] = ms
            if ms < best_ms:
                best, best_ms = c, ms
        return best, timings, count or 0

    @staticmethod
    def _device_runner(R, S, eps2, mode, screen):
        def run(c: Choice):
            res = api.join_result(R, S, eps2=eps2, mode=mode, screen=screen, **c.kwargs())
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
        """Time every applicable choice on a row sample and record the fastest; returns
        (choice, key, timings in ms per choice)."""
        Rt, _ = api._as_device(R, screen == "int8limb")
        St = None if S is None else api._as_device(S, screen == "int8limb")[0]
        Rs, Ss, scale = self._sample(Rt, St, mode, sample_rows)
        d = Rt.shape[1]
        best, timings, count = self.pick(candidates(d, screen, mode),
                                         self._device_runner(Rs, Ss, eps2, mode, screen), reps)
        per_row = count / max(1, Rs.shape[0]) * scale
        key = tune_key(d, _dtype(Rt), screen, mode, Rt.shape[0], Rt.shape[0] if St is None else St.shape[0], per_row)
        self.record(key, best, timings)
        return best, key, timings

    def key_for(self, R, S, eps2: float, mode: str, screen: str, probe_rows: int = 512) -> str:
        """Key of the full join, with the selectivity measured on a small row sample."""
        Rt, _ = api._as_device(R, screen == "int8limb")
        St = None if S is None else api._as_device(S, screen == "int8limb")[0]
        Rs, Ss, scale = self._sample(Rt, St, mode, probe_rows)
        res = api.join_result(Rs, Ss, eps2=eps2, mode=mode, screen=screen)
        per_row = res.count / max(1, Rs.shape[0]) * scale
        return tune_key(Rt.shape[1], _dtype(Rt), screen, mode, Rt.shape[0],
                        Rt.shape[0] if St is None else St.shape[0], per_row)

    def join(self, R, S=None, eps=None, *, eps2=None, mode: str = "rs", screen: str = "bf16",
             sample_rows: int = 4096) -> api.Result:
        """Run the join with the table's choice for its key, tuning first on a miss."""
        T = api._threshold(eps, eps2)
        key = self.key_for(R, S, T, mode, screen)
        choice = self.lookup(key)
        if choice is None:   # the tuning sample may bucket its selectivity differently: keep both keys
            choice, _, timings = self.tune(R, S, T, mode, screen, sample_rows)
            self.record(key, choice, timings)
        return api.join_result(R, S, eps2=T, mode=mode, screen=screen, **choice.kwargs())


def _dtype(t: torch.Tensor) -> str:
    return "i16" if t.dtype == torch.int16 else "f32"


__all__ = ["Choice", "Tuner", "candidates", "tune_key", "CHUNK_ITEMS"]
