"""CPU oracle for the certified exact epsilon-join -- TEST INFRASTRUCTURE.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline
leg may import this package, and only as the checker (or the timed CPU
baseline).  The product path (``tensorjoin_variants_b200``) never imports it.

Three restatements of the reference's exact CPU predicate live here:

* ``join_f32`` / ``join_i16``: the C oracle of record (``oracle.c``), FP64
  direct difference with a fixed sequential k order and no FMA contraction,
  multithreaded over row blocks.  The GPU FP64 refinement reproduces exactly
  this order, so the GPU pair set is compared with it bit for bit.
* ``py_join``: pure-Python loops in the same order, for tiny cases; it pins
  the C build (same IEEE operations, same order, same result).
* ``scipy_join``: the reference's own exact CPU path,
  ``scipy.spatial.distance.cdist(R64, S64, "sqeuclidean") <= T``
  (tensorjoin_20260902_certified_exact_join/src/prepare_g2_cifar.py:189,
  src/build_g4b_exact_oracles.py:142; R-S einsum variant src/run_d1_triton.py:69-79).
  SciPy's internal summation order is compiled third-party code, so this is a
  cross-check: it may differ from the sequential order only at FP64 ties.

Output of every join is the ascending uint64 array of canonical keys
``i * n_cols + j`` (src/g2b_public_common.py:106-143).  Modes: ``"rs"``
(all i, j), ``"upper"`` (self-join, i < j), ``"directed"`` (self-join, all
i, j including i == j).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "_build" / "liboracle.so"
MODES = {"rs": 0, "upper": 1, "directed": 2}
_lib = None


def build() -> Path:
    """Compile the C oracle with its Makefile (``-ffp-contract=off``)."""
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            build()
        L = C.CDLL(str(LIB_PATH))
        P = C.c_void_p
        L.oracle_join_f32.argtypes = [P, C.c_int64, P, C.c_int64, C.c_int, C.c_double, C.c_int, C.c_int,
                                      C.POINTER(C.c_void_p), C.POINTER(C.c_int64)]
        L.oracle_join_f32.restype = C.c_int
        L.oracle_join_i16.argtypes = [P, C.c_int64, P, C.c_int64, C.c_int, C.c_int64, C.c_int, C.c_int,
                                      C.POINTER(C.c_void_p), C.POINTER(C.c_int64)]
        L.oracle_join_i16.restype = C.c_int
        L.oracle_free.argtypes = [P]
        L.oracle_pair_d2_f32.argtypes = [P, P, C.c_int, P, P, C.c_int64, P]
        L.oracle_row_counts_f32.argtypes = [P, C.c_int64, P, C.c_int64, C.c_int, C.c_double, P, C.c_int64, P]
        L.oracle_row_counts_f32.restype = C.c_int
        L.oracle_pair_d2_f32_mt.argtypes = [P, P, C.c_int, P, P, C.c_int64, P, C.c_int]
        L.oracle_pair_d2_f32_mt.restype = C.c_int
        L.oracle_pair_d2_i16_mt.argtypes = [P, P, C.c_int, P, P, C.c_int64, P, C.c_int]
        L.oracle_pair_d2_i16_mt.restype = C.c_int
        L.oracle_abi_version.restype = C.c_int
        if L.oracle_abi_version() != 2:
            raise RuntimeError(f"{LIB_PATH} is a stale build: run oracle.build()")
        _lib = L
    return _lib


def default_threads() -> int:
    return max(1, len(os.sched_getaffinity(0)))


def _collect(rc, ptr, count):
    if rc != 0:
        raise RuntimeError(f"oracle failed with code {rc}")
    n = int(count.value)
    if n == 0:
        lib().oracle_free(ptr)
        return np.empty(0, dtype=np.uint64)
    buf = (C.c_uint64 * n).from_address(ptr.value)
    out = np.frombuffer(buf, dtype=np.uint64).copy()
    lib().oracle_free(ptr)
    return out


def join_f32(R: np.ndarray, S: np.ndarray | None, T: float, mode: str = "rs", threads: int | None = None) -> np.ndarray:
    """Sorted canonical keys of all pairs with sequential FP64 d2 <= T (FP32 inputs)."""
    R = np.ascontiguousarray(R, dtype=np.float32)
    S = R if S is None else np.ascontiguousarray(S, dtype=np.float32)
    if mode != "rs" and S is not R and not np.array_equal(R, S):
        raise ValueError("self-join modes need S == R")
    ptr, cnt = C.c_void_p(), C.c_int64()
    rc = lib().oracle_join_f32(R.ctypes.data, R.shape[0], S.ctypes.data, S.shape[0], R.shape[1], float(T),
                               MODES[mode], threads or default_threads(), C.byref(ptr), C.byref(cnt))
    return _collect(rc, ptr, cnt)


def join_i16(R: np.ndarray, S: np.ndarray | None, T: int, mode: str = "rs", threads: int | None = None) -> np.ndarray:
    """Sorted canonical keys of all pairs with exact integer d2 <= T (int16 inputs)."""
    R = np.ascontiguousarray(R, dtype=np.int16)
    S = R if S is None else np.ascontiguousarray(S, dtype=np.int16)
    ptr, cnt = C.c_void_p(), C.c_int64()
    rc = lib().oracle_join_i16(R.ctypes.data, R.shape[0], S.ctypes.data, S.shape[0], R.shape[1], int(T),
                               MODES[mode], threads or default_threads(), C.byref(ptr), C.byref(cnt))
    return _collect(rc, ptr, cnt)


def pair_d2(R: np.ndarray, S: np.ndarray, i: np.ndarray, j: np.ndarray) -> np.ndarray:
    """Sequential-order FP64 squared distances for explicit pairs (R[i], S[j])."""
    R = np.ascontiguousarray(R, dtype=np.float32)
    S = np.ascontiguousarray(S, dtype=np.float32)
    i = np.ascontiguousarray(i, dtype=np.int64)
    j = np.ascontiguousarray(j, dtype=np.int64)
    out = np.empty(len(i), dtype=np.float64)
    lib().oracle_pair_d2_f32(R.ctypes.data, S.ctypes.data, R.shape[1], i.ctypes.data, j.ctypes.data, len(i),
                             out.ctypes.data)
    return out


def pair_d2_mt(R: np.ndarray, S: np.ndarray, i: np.ndarray, j: np.ndarray, threads: int | None = None) -> np.ndarray:
    """Squared distances of explicit pairs (R[i], S[j]) over host threads: sequential-order FP64 for
    FP32 rows (float64 result), exact int64 for int16 rows (int64 result)."""
    is_int = np.asarray(R).dtype == np.int16
    dt = np.int16 if is_int else np.float32
    R = np.ascontiguousarray(R, dtype=dt)
    S = np.ascontiguousarray(S, dtype=dt)
    i = np.ascontiguousarray(i, dtype=np.int64)
    j = np.ascontiguousarray(j, dtype=np.int64)
    if len(i) != len(j):
        raise ValueError("i and j differ in length")
    if len(i) and (i.min() < 0 or i.max() >= R.shape[0] or j.min() < 0 or j.max() >= S.shape[0]):
        raise IndexError("pair index out of range")
    out = np.empty(len(i), dtype=np.int64 if is_int else np.float64)
    fn = lib().oracle_pair_d2_i16_mt if is_int else lib().oracle_pair_d2_f32_mt
    rc = fn(R.ctypes.data, S.ctypes.data, R.shape[1], i.ctypes.data, j.ctypes.data, len(i), out.ctypes.data,
            threads or default_threads())
    if rc != 0:
        raise RuntimeError(f"oracle failed with code {rc}")
    return out


def row_counts(R: np.ndarray, S: np.ndarray, T: float, rows: np.ndarray) -> np.ndarray:
    """Number of S rows within T of each selected R row (sequential FP64 order)."""
    R = np.ascontiguousarray(R, dtype=np.float32)
    S = np.ascontiguousarray(S, dtype=np.float32)
    rows = np.ascontiguousarray(rows, dtype=np.int64)
    out = np.empty(len(rows), dtype=np.int64)
    lib().oracle_row_counts_f32(R.ctypes.data, R.shape[0], S.ctypes.data, S.shape[0], R.shape[1], float(T),
                                rows.ctypes.data, len(rows), out.ctypes.data)
    return out


def py_join(R, S, T, mode: str = "rs") -> np.ndarray:
    """Pure-Python sequential loops (tiny inputs only): pins the C oracle."""
    R = np.asarray(R, dtype=np.float32)
    S = R if S is None else np.asarray(S, dtype=np.float32)
    nS = S.shape[0]
    keys = []
    for i in range(R.shape[0]):
        x = [float(v) for v in R[i]]
        j0 = i + 1 if mode == "upper" else 0
        for j in range(j0, nS):
            acc = 0.0
            for k, yv in enumerate(S[j]):
                t = x[k] - float(yv)
                acc = acc + t * t
            if acc <= T:
                keys.append(i * nS + j)
    return np.array(keys, dtype=np.uint64)


def scipy_join(R: np.ndarray, S: np.ndarray | None, T: float, mode: str = "rs", block: int = 512) -> np.ndarray:
    """The reference's CPU exact path: SciPy cdist 'sqeuclidean' on FP64-widened rows, then <= T."""
    from scipy.spatial.distance import cdist

    R64 = np.asarray(R, dtype=np.float32).astype(np.float64)
    S64 = R64 if S is None else np.asarray(S, dtype=np.float32).astype(np.float64)
    nS = S64.shape[0]
    parts = []
    for r0 in range(0, R64.shape[0], block):
        d2 = cdist(R64[r0:r0 + block], S64, "sqeuclidean")
        ii, jj = np.nonzero(d2 <= T)
        ii = ii + r0
        if mode == "upper":
            keep = jj > ii
            ii, jj = ii[keep], jj[keep]
        parts.append(ii.astype(np.uint64) * np.uint64(nS) + jj.astype(np.uint64))
    return np.concatenate(parts) if parts else np.empty(0, dtype=np.uint64)


def _scipy_rows(args):
    R, S, T, r0, r1 = args
    from scipy.spatial.distance import cdist

    d2 = cdist(R[r0:r1].astype(np.float64), S.astype(np.float64), "sqeuclidean")
    return int(np.count_nonzero(d2 <= T))


def scipy_count_parallel(R: np.ndarray, S: np.ndarray, T: float, processes: int, rows_per_task: int = 64) -> int:
    """Count pairs with SciPy cdist over row blocks in ``processes`` spawned workers (CPU baseline)."""
    import multiprocessing as mp

    tasks = [(R, S, T, r0, min(r0 + rows_per_task, R.shape[0])) for r0 in range(0, R.shape[0], rows_per_task)]
    ctx = mp.get_context("spawn")
    with ctx.Pool(processes) as pool:
        return int(sum(pool.map(_scipy_rows, tasks)))


def keys_to_ij(keys: np.ndarray, n_cols: int) -> tuple[np.ndarray, np.ndarray]:
    keys = np.asarray(keys, dtype=np.uint64)
    return (keys // np.uint64(n_cols)).astype(np.int64), (keys % np.uint64(n_cols)).astype(np.int64)


def directed_from_upper(upper: np.ndarray, n: int) -> np.ndarray:
    """Expand upper (i < j) keys to the directed canonical set with the n self pairs
    (the reference's mirror step, tensorjoin_20260908_output_audit/src/output.cu:8-18)."""
    i, j = keys_to_ij(upper, n)
    diag = np.arange(n, dtype=np.uint64)
    out = np.concatenate([upper.astype(np.uint64), j.astype(np.uint64) * np.uint64(n) + i.astype(np.uint64),
                          diag * np.uint64(n) + diag])
    out.sort()
    return out


# ---------------------------------------------------------------- CPU baseline timing (SciPy, shared memory)
_SHM = {}


def _attach(names):
    from multiprocessing import shared_memory

    for key, (name, shape, dtype) in names.items():
        shm = shared_memory.SharedMemory(name=name)
        _SHM[key] = (shm, np.ndarray(shape, dtype=dtype, buffer=shm.buf))
    # the reference widens both sides to FP64 once (src/prepare_g2_cifar.py:189); done at worker start-up
    _SHM["S64"] = (None, _SHM["S"][1].astype(np.float64))


def _count_block(args):
    r0, r1, T = args
    from scipy.spatial.distance import cdist

    R = _SHM["R"][1]
    d2 = cdist(R[r0:r1].astype(np.float64), _SHM["S64"][1], "sqeuclidean")
    return int(np.count_nonzero(d2 <= T))


def scipy_rate(R_rows: np.ndarray, S: np.ndarray, T: float, processes: int, rows_per_task: int = 4,
               repeats: int = 1, context: str = "spawn"):
    """Time the reference's CPU exact path (SciPy cdist 'sqeuclidean' + ``<= T``) on ``R_rows`` x all of S.

    Rows are spread over ``processes`` workers (spawned by default, so it is safe after CUDA init);
    S lives in shared memory.  Returns (pairs evaluated per repeat, list of seconds per repeat, count).
    """
    import multiprocessing as mp
    import time
    from multiprocessing import shared_memory

    R_rows = np.ascontiguousarray(R_rows, dtype=np.float32)
    S = np.ascontiguousarray(S, dtype=np.float32)
    shms, names = [], {}
    for key, arr in (("R", R_rows), ("S", S)):
        shm = shared_memory.SharedMemory(create=True, size=max(arr.nbytes, 1))
        np.ndarray(arr.shape, dtype=arr.dtype, buffer=shm.buf)[...] = arr
        shms.append(shm)
        names[key] = (shm.name, arr.shape, arr.dtype.str)
    try:
        ctx = mp.get_context(context)
        tasks = [(r0, min(r0 + rows_per_task, len(R_rows)), float(T)) for r0 in range(0, len(R_rows), rows_per_task)]
        secs, count = [], 0
        with ctx.Pool(processes, initializer=_attach, initargs=(names,)) as pool:
            pool.map(_count_block, [(0, 1, float(T))] * processes)   # warm the workers (imports, page-in)
            for _ in range(repeats):
                t0 = time.perf_counter()
                count = sum(pool.map(_count_block, tasks))
                secs.append(time.perf_counter() - t0)
        return len(R_rows) * len(S), secs, count
    finally:
        for shm in shms:
            shm.close()
            shm.unlink()
