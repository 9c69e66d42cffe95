"""Python drop-in for the certified exact epsilon-join.

``join(R, S, eps)`` and ``self_join(X, eps)`` return the pair set
``{(i, j) : sum_k (double(R[i,k]) - double(S[j,k]))^2 <= eps^2}`` (FP64, sequential
k order; exact integers for int16 input) as two int64 arrays sorted by (i, j).
``build_index(X, eps)`` exposes the Morton-grid index.  Inputs may be CUDA
tensors (results stay on the device) or host arrays / CPU tensors (inputs are
copied in on the current stream and results come back to the host).

The reference has no library API for this path; these functions give its
script-level contract a callable form: FP32 rows in, sorted canonical ids out
(tensorjoin_20260902_certified_exact_join/src/g2b_public_common.py:97-143),
self-join and R-S modes (src/run_g2a2_tensorjoin_triangular.py:42-141,
src/run_d1_triton.py:110-248), canonical keys ``i * n_cols + j`` and the
GDS-style neighbour table (adapters/gds_g2a/main.cu:488-510).
Every computation runs in libtensorjoin.so on the GPU; there is no CPU path.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass

import numpy as np
import torch

from . import _lib
from ._lib import MODE, SCREEN, check, lib

__all__ = ["join", "self_join", "join_result", "build_index", "Result", "Index", "join_batched",
           "join_batched_result", "BatchResult"]


def _stream_ptr() -> int:
    return torch.cuda.current_stream().cuda_stream


def _as_device(x, allow_int16: bool):
    """Return (device tensor, was_host).  Host inputs are copied in on the current stream."""
    was_host = True
    if isinstance(x, torch.Tensor):
        t = x
        if t.is_cuda:
            was_host = False
        else:
            t = t.to("cuda", non_blocking=t.is_pinned())
    else:
        arr = np.asarray(x)
        if arr.dtype not in (np.float32, np.int16):
            arr = arr.astype(np.float32)
        t = torch.from_numpy(np.ascontiguousarray(arr)).to("cuda")
    if t.dim() != 2:
        raise ValueError("inputs must be 2-D [rows, dims]")
    if t.dtype not in (torch.float32, torch.int16):
        raise TypeError(f"unsupported dtype {t.dtype}: use float32 (or int16 for int14 data)")
    if t.dtype == torch.int16 and not allow_int16:
        raise TypeError("int16 input needs screen='int8limb'")
    return t.contiguous(), was_host


def _threshold(eps, eps2) -> float:
    if eps2 is not None:
        return float(eps2)
    if eps is None:
        raise ValueError("give eps or eps2")
    e = float(eps)
    if not (e >= 0) or math.isinf(e):
        raise ValueError("eps must be finite and >= 0")
    return e * e


class Result:
    """Owns a tj_result handle: sorted canonical pairs on the device plus statistics."""

    def __init__(self, handle: C.c_void_p, n_rows: int, n_cols: int, host: bool, keepalive=()):
        self._h = handle
        self.n_rows, self.n_cols, self.host = n_rows, n_cols, host
        self._keep = keepalive

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            lib().tj_result_free(h)
            self._h = None

    @property
    def count(self) -> int:
        return int(lib().tj_result_count(self._h))

    @property
    def stats(self) -> dict:
        s = _lib.Stats()
        check(lib().tj_result_stats(self._h, C.byref(s)))
        return s.as_dict()

    def _out(self, *ts):
        """Host callers get host tensors: copied into pinned buffers on the current stream (one
        synchronisation for all of them), which runs at the link's rate instead of staging
        through pageable memory."""
        if not self.host:
            return ts
        outs = tuple(torch.empty(t.shape, dtype=t.dtype, pin_memory=True) for t in ts)
        for o, t in zip(outs, ts):
            o.copy_(t, non_blocking=True)
        torch.cuda.current_stream().synchronize()
        return outs

    def pairs(self):
        n = self.count
        i = torch.empty(n, dtype=torch.int64, device="cuda")
        j = torch.empty(n, dtype=torch.int64, device="cuda")
        if n:
            check(lib().tj_result_pairs(self._h, C.c_void_p(i.data_ptr()), C.c_void_p(j.data_ptr()),
                                        C.c_void_p(_stream_ptr())))
        return self._out(i, j)

    def keys(self):
        """Canonical keys i * n_cols + j (int64 tensor holding the uint64 values, ascending)."""
        n = self.count
        k = torch.empty(n, dtype=torch.int64, device="cuda")
        if n:
            check(lib().tj_result_keys(self._h, C.c_void_p(k.data_ptr()), C.c_void_p(_stream_ptr())))
        return self._out(k)[0]

    def stage_keys(self, stage: int):
        """The screen's own decisions (join run with ``stage_keys=True``): stage 0 = pairs it accepted
        by its certificate alone, stage 1 = its band, as sorted canonical keys (i < j for self-joins)."""
        n = C.c_int64()
        check(lib().tj_result_stage_keys(self._h, int(stage), None, C.byref(n), C.c_void_p(_stream_ptr())))
        k = torch.empty(n.value, dtype=torch.int64, device="cuda")
        if n.value:
            check(lib().tj_result_stage_keys(self._h, int(stage), C.c_void_p(k.data_ptr()), C.byref(n),
                                             C.c_void_p(_stream_ptr())))
        return self._out(k)[0]

    def neighbor_table(self):
        """GDS-style output: neighbour counts per row and the flat, row-ordered neighbour list."""
        counts = torch.empty(self.n_rows, dtype=torch.int32, device="cuda")
        flat = torch.empty(self.count, dtype=torch.int64, device="cuda")
        check(lib().tj_result_neighbor_table(self._h, C.c_void_p(counts.data_ptr()), C.c_void_p(flat.data_ptr()),
                                             C.c_void_p(_stream_ptr())))
        return self._out(counts, flat)


def _run(R, S, eps, eps2, mode: str, screen: str, capacity: int, chunk_items: int, flags: int = 0,
         k_block: int = 0, stages: int = 0) -> Result:
    if screen not in SCREEN:
        raise ValueError(f"screen must be one of {sorted(SCREEN)}")
    Rt, host = _as_device(R, screen == "int8limb")
    if mode == "rs":
        St, host_s = _as_device(S, screen == "int8limb")
        host = host and host_s
        if St.shape[1] != Rt.shape[1]:
            raise ValueError("R and S must have the same number of dimensions")
        if St.dtype != Rt.dtype:
            raise TypeError("R and S must have the same dtype")
    else:
        St = Rt
    T = _threshold(eps, eps2)
    dtype = _lib.DTYPE["i16"] if Rt.dtype == torch.int16 else _lib.DTYPE["f32"]
    opt = _lib.Options(int(capacity), int(chunk_items), int(flags), int(k_block), int(stages))
    h = C.c_void_p()
    check(lib().tj_join(C.c_void_p(Rt.data_ptr()), Rt.shape[0], C.c_void_p(St.data_ptr()), St.shape[0],
                        Rt.shape[1], dtype, T, MODE[mode], SCREEN[screen], C.byref(opt), C.byref(h),
                        C.c_void_p(_stream_ptr())))
    return Result(h, Rt.shape[0], St.shape[0] if mode == "rs" else Rt.shape[0], host, keepalive=(Rt, St))


FRAME_FLAGS = {"auto": 0, "axes": _lib.FLAG_FRAME_AXES, "pca": _lib.FLAG_FRAME_PCA}


def join_result(R, S, eps=None, *, eps2=None, mode: str = "rs", screen: str = "bf16", capacity: int = 0,
                chunk_items: int = 0, screen_diag: bool = False, cta_pair: bool = True,
                index_frame: str = "auto", band_fp32: bool = False, i8_four_products: bool = False,
                guards: bool = False, stage_keys: bool = False, screen_times: bool = False,
                k_block: int = 0, stages: int = 0, half_pack: bool = True) -> Result:
    """Run a join and return the Result handle (pairs, keys, neighbour table, statistics).

    ``screen_diag=True`` also samples 64 tile pairs of the tensor-core screen and reports, in
    ``stats``, the screen's largest distance error against sequential FP64 distances and that
    error relative to the certified radius (must stay below 1).  ``cta_pair=False`` keeps the
    one-SM screen where the CTA-pair screen would run (``stats["screen_pair"]`` says which ran).
    ``index_frame`` picks the cells rows are sorted by before tiling: "auto", "axes" (the 8
    highest-variance input dimensions) or "pca" (the top 8 principal directions, 9 <= d <= 128);
    ``stats["index_frame"]`` is 1 where the principal-direction cells were used.
    ``band_fp32=True`` decides band pairs by a certified FP32 sum first and sends only the rest to
    the FP64 terminal (``stats["band_fp64"]`` counts those).  ``i8_four_products=True`` makes the
    int8-limb screen issue all four limb products and decide every pair inside the screen, instead of
    the high-limb product plus an exact integer refinement of the undecided band.  ``guards=True``
    checks guard regions after every output buffer (an overwrite fails the join); ``stage_keys=True``
    keeps the screen's certified accepts and its band for ``Result.stage_keys``.  ``k_block`` (16, 32
    or 64 elements of K per stage) and ``stages`` (operand stages in flight) are tile-shape knobs of
    the 16-bit screens for the autotuner; 0 keeps the library's choice.  ``half_pack=False`` makes
    the one-SM screen issue both 128-row halves of every candidate tile pair (by default dead halves
    are dropped after a half-tile bound test).  ``screen="auto"`` takes the
    screen and knobs from the committed B200 tuning table (``autotune.default_table``) for this
    workload's key (d, size, selectivity measured on a 512-row probe), BF16 hi/lo on a miss."""
    if mode not in MODE:
        raise ValueError(f"mode must be one of {sorted(MODE)}")
    if index_frame not in FRAME_FLAGS:
        raise ValueError(f"index_frame must be one of {sorted(FRAME_FLAGS)}")
    if screen == "auto":   # the committed tuning table's choice for this workload (library defaults on a miss)
        from . import autotune

        choice, _ = autotune.default_table().choose(R, S, _threshold(eps, eps2), mode, "auto", tune_on_miss=False)
        kw = choice.kwargs()
        return join_result(R, S, eps2=_threshold(eps, eps2), mode=mode, screen=choice.screen_for("bf16x3"),
                           capacity=capacity, chunk_items=chunk_items or kw["chunk_items"], screen_diag=screen_diag,
                           cta_pair=cta_pair and kw["cta_pair"],
                           index_frame=index_frame if index_frame != "auto" else kw["index_frame"],
                           band_fp32=band_fp32 or kw["band_fp32"], guards=guards, stage_keys=stage_keys,
                           screen_times=screen_times, k_block=k_block or kw["k_block"], stages=stages or kw["stages"],
                           half_pack=half_pack and kw["half_pack"],
                           i8_four_products=i8_four_products or kw["i8_four_products"])
    flags = (_lib.FLAG_SCREEN_DIAG if screen_diag else 0) | (0 if cta_pair else _lib.FLAG_SCREEN_1SM)
    flags |= FRAME_FLAGS[index_frame] | (_lib.FLAG_BAND_FP32 if band_fp32 else 0)
    flags |= _lib.FLAG_I8_FOUR_PRODUCTS if i8_four_products else 0
    flags |= (_lib.FLAG_GUARDS if guards else 0) | (_lib.FLAG_STAGE_KEYS if stage_keys else 0)
    flags |= _lib.FLAG_SCREEN_TIMES if screen_times else 0
    flags |= 0 if half_pack else _lib.FLAG_WHOLE_TILES
    return _run(R, S, eps, eps2, mode, screen, capacity, chunk_items, flags, k_block, stages)


def join(R, S, eps=None, *, eps2=None, screen: str = "bf16", return_stats: bool = False, **kw):
    """R-S epsilon-join: sorted (i, j) with FP64 direct-difference distance <= eps
    (``screen="auto"``: the tuned choice, see ``join_result``)."""
    res = join_result(R, S, eps, eps2=eps2, mode="rs", screen=screen, **kw)
    i, j = res.pairs()
    return (i, j, res.stats) if return_stats else (i, j)


def self_join(X, eps=None, *, eps2=None, mode: str = "upper", screen: str = "bf16", return_stats: bool = False,
              **kw):
    """Self-join: mode 'upper' gives i < j; 'directed' gives all (i, j) incl. the N self pairs."""
    if mode not in ("upper", "directed"):
        raise ValueError("self_join mode must be 'upper' or 'directed'")
    res = join_result(X, None, eps, eps2=eps2, mode=mode, screen=screen, **kw)
    i, j = res.pairs()
    return (i, j, res.stats) if return_stats else (i, j)


@dataclass
class Index:
    """Morton-grid index of one point set (device tensors)."""
    perm: torch.Tensor         # [n] int32: sorted position -> input row
    keys: torch.Tensor         # [n] int64: Morton keys, ascending
    cell_start: torch.Tensor   # [n_cells + 1] int32: prefix offsets of the cells in sorted order
    tile_pairs: torch.Tensor   # [P, 2] int32: candidate (128-row tile, 256-row tile) pairs at eps
    n_tiles: int


def build_index(X, eps=None, *, eps2=None) -> Index:
    """Build the GPU Morton-grid index of X (cells, prefix offsets, candidate tile pairs at eps)."""
    Xt, _ = _as_device(X, True)
    T = _threshold(eps, eps2)
    dtype = _lib.DTYPE["i16"] if Xt.dtype == torch.int16 else _lib.DTYPE["f32"]
    h = C.c_void_p()
    check(lib().tj_index_build(C.c_void_p(Xt.data_ptr()), Xt.shape[0], Xt.shape[1], dtype, T, C.byref(h),
                               C.c_void_p(_stream_ptr())))
    try:
        nc, nt, npairs = C.c_int64(), C.c_int64(), C.c_int64()
        check(lib().tj_index_info(h, C.byref(nc), C.byref(nt), C.byref(npairs)))
        n = Xt.shape[0]
        perm = torch.empty(n, dtype=torch.int32, device="cuda")
        keys = torch.empty(n, dtype=torch.int64, device="cuda")
        cs = torch.empty(nc.value + 1, dtype=torch.int32, device="cuda")
        tp = torch.empty((npairs.value, 2), dtype=torch.int32, device="cuda")
        check(lib().tj_index_copy(h, C.c_void_p(perm.data_ptr()), C.c_void_p(keys.data_ptr()),
                                  C.c_void_p(cs.data_ptr()), C.c_void_p(tp.data_ptr() if npairs.value else 0),
                                  C.c_void_p(_stream_ptr())))
        torch.cuda.current_stream().synchronize()
    finally:
        lib().tj_index_free(h)
    return Index(perm, keys, cs, tp, int(nt.value))


class BatchResult(Result):
    """Result of a batched join: all joins' pairs in one sorted array plus per-join ranges."""

    def __init__(self, handle, njoins: int, host: bool, keepalive=()):
        super().__init__(handle, 0, 0, host, keepalive)
        self.njoins = njoins

    def offsets(self):
        offs = (C.c_int64 * (self.njoins + 1))()
        check(lib().tj_batch_offsets(self._h, offs))
        return [int(v) for v in offs]

    def pairs(self):
        n = self.count
        i = torch.empty(n, dtype=torch.int64, device="cuda")
        j = torch.empty(n, dtype=torch.int64, device="cuda")
        if n:
            check(lib().tj_batch_pairs(self._h, C.c_void_p(i.data_ptr()), C.c_void_p(j.data_ptr()),
                                       C.c_void_p(_stream_ptr())))
        return self._out(i, j)

    def split(self):
        """[(i, j)] per join, in join order (local row ids of each join's R and S)."""
        i, j = self.pairs()
        o = self.offsets()
        return [(i[o[k]:o[k + 1]], j[o[k]:o[k + 1]]) for k in range(self.njoins)]


def _host_views_to_device(xs):
    """Host tensors that are contiguous 2-D views of one host array (the rows of many joins in a few
    large arrays) go to the device in one copy per array: the span the views cover is copied once
    and each view becomes the matching device view, so views that lie back to back on the host stay
    back to back on the device (the batched join then reads them in place).  Returns, per input,
    ``(device tensor, True)`` or None for inputs left to ``_as_device``."""
    out = [None] * len(xs)
    groups: dict = {}
    for q, x in enumerate(xs):
        if (isinstance(x, torch.Tensor) and not x.is_cuda and x.dim() == 2 and x.is_contiguous()
                and x.dtype == torch.float32):
            groups.setdefault(x.untyped_storage().data_ptr(), []).append(q)
    for idx in groups.values():
        if len(idx) < 2:
            continue
        first = xs[idx[0]]
        lo = min(xs[q].storage_offset() for q in idx)
        hi = max(xs[q].storage_offset() + xs[q].numel() for q in idx)
        span = torch.empty(0, dtype=first.dtype).set_(first.untyped_storage(), lo, (hi - lo,), (1,))
        dev = span.to("cuda", non_blocking=span.is_pinned())
        for q in idx:
            x = xs[q]
            o = x.storage_offset() - lo
            out[q] = (dev[o:o + x.numel()].view(x.shape), True)
    return out


def join_batched_result(joins, screen: str = "bf16", capacity: int = 0, chunk_items: int = 0,
                        index_frame: str = "auto", band_fp32: bool = False,
                        screen_diag: bool = False, screen_times: bool = False, guards: bool = False,
                        k_block: int = 0, stages: int = 0, cta_pair: bool = True,
                        half_pack: bool = True) -> BatchResult:
    """Run many independent R-S joins [(R, S, eps), ...] in one batched pass (one screen launch).
    ``index_frame``, ``band_fp32``, ``screen_diag`` and ``guards`` as in ``join_result`` (packed joins
    keep input-dimension cells under "auto").  ``screen_times=True`` stamps each join's first and last
    chunk inside the screen launch and each CTA's end (``stats["join_span_ms_p50"]``, ``_p99``,
    ``_max`` and ``stats["screen_cta_tail_ms"]``)."""
    if index_frame not in FRAME_FLAGS:
        raise ValueError(f"index_frame must be one of {sorted(FRAME_FLAGS)}")
    descs = (_lib.BatchJoin * len(joins))()
    keep = []
    host = True
    moved = _host_views_to_device([x for R, S, _ in joins for x in (R, S)])
    for k, (R, S, eps) in enumerate(joins):
        Rt, hr = moved[2 * k] if moved[2 * k] is not None else _as_device(R, False)
        St, hs = moved[2 * k + 1] if moved[2 * k + 1] is not None else _as_device(S, False)
        host = host and hr and hs
        keep += [Rt, St]
        descs[k] = _lib.BatchJoin(Rt.data_ptr(), St.data_ptr(), Rt.shape[0], St.shape[0], Rt.shape[1], 0,
                                  _threshold(eps, None))
    h = C.c_void_p()
    flags = FRAME_FLAGS[index_frame] | (_lib.FLAG_BAND_FP32 if band_fp32 else 0)
    flags |= _lib.FLAG_SCREEN_DIAG if screen_diag else 0
    flags |= (_lib.FLAG_SCREEN_TIMES if screen_times else 0) | (_lib.FLAG_GUARDS if guards else 0)
    flags |= 0 if cta_pair else _lib.FLAG_SCREEN_1SM
    flags |= 0 if half_pack else _lib.FLAG_WHOLE_TILES
    opt = _lib.Options(int(capacity), int(chunk_items), flags, int(k_block), int(stages))
    check(lib().tj_join_batched(descs, len(joins), SCREEN[screen], C.byref(opt), C.byref(h),
                                C.c_void_p(_stream_ptr())))
    return BatchResult(h, len(joins), host, keepalive=tuple(keep))


def join_batched(joins, screen: str = "bf16", **kw):
    """Many independent R-S joins [(R, S, eps), ...] in one batched pass; returns [(i, j), ...]."""
    return join_batched_result(joins, screen=screen, **kw).split()
