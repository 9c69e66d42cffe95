"""ctypes binding of libtensorjoin.so (the C ABI declared in include/tensorjoin.h).

The style follows the reference's ctypes wrappers of its native stages
(tensorjoin_20260908_output_audit/src/common.py:24-39,
adapters/gds_g2a/gdsjoingpu.py:146-232): argtypes declared once, status codes
turned into exceptions.  There is no fallback: if the library is missing the
import fails loudly.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libtensorjoin.so"

TJ_OK = 0
ERRORS = {
    -1: "TJ_ERR_INVALID", -2: "TJ_ERR_CUDA", -3: "TJ_ERR_INPUT", -4: "TJ_ERR_RANGE",
    -5: "TJ_ERR_TIMEOUT", -6: "TJ_ERR_NOMEM", -7: "TJ_ERR_UNSUPPORTED",
}
DTYPE = {"f32": 0, "i16": 1}
MODE = {"rs": 0, "upper": 1, "directed": 2}
SCREEN = {"plain": 0, "bf16": 1, "fp16": 2, "int8limb": 3, "bf16x3": 4, "fp16x3": 5}
FLAG_SCREEN_DIAG = 1
FLAG_SCREEN_1SM = 2
FLAG_FRAME_AXES = 4
FLAG_FRAME_PCA = 8
FLAG_BAND_FP32 = 16
FLAG_I8_FOUR_PRODUCTS = 32
FLAG_GUARDS = 64
FLAG_STAGE_KEYS = 128
FLAG_SCREEN_TIMES = 256
FLAG_WHOLE_TILES = 512

# Every symbol include/tensorjoin.h declares (checked by the CPU test suite).
EXPORTS = [
    "tj_join", "tj_result_count", "tj_result_stats", "tj_result_pairs", "tj_result_keys",
    "tj_result_neighbor_table", "tj_result_free", "tj_index_build", "tj_index_info", "tj_index_copy",
    "tj_index_free", "tj_join_batched", "tj_batch_offsets", "tj_batch_pairs", "tj_last_error_string",
    "tj_version", "tj_device_sm_count", "tj_kernel_launches", "tj_sort_keys_noalloc",
    "tj_pool_usage", "tj_pool_reserve", "tj_pool_trim", "tj_set_wait_limit", "tj_result_stage_keys",
]


class TJError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")
        self.code = code


class Options(C.Structure):
    _fields_ = [("initial_capacity", C.c_int64), ("chunk_items", C.c_int32), ("flags", C.c_int32),
                ("k_block", C.c_int32), ("stages", C.c_int32)]


class Stats(C.Structure):
    _fields_ = [(n, C.c_int64) for n in (
        "n_rows", "n_cols", "pairs_all", "tile_pairs", "pairs_screened", "screen_accept", "band",
        "refine_accept", "rare_checks", "result_pairs", "retries")] + [(n, C.c_double) for n in (
        "ms_index", "ms_candidates", "ms_screen", "ms_refine", "ms_sort", "ms_total", "screen_ops",
        "screen_max_abs_err", "screen_err_over_bound")] + [("screen_err_pairs", C.c_int64), ("screen_pair", C.c_int64),
                                                   ("index_frame", C.c_int64), ("band_fp64", C.c_int64),
                                                   ("screen_ops_issued", C.c_double)] + [
        (n, C.c_double) for n in ("screen_cta_tail_ms", "join_span_ms_p50", "join_span_ms_p99", "join_span_ms_max",
                                  "screen_prod_stage_wait", "screen_prod_meta_wait", "screen_mma_operand_wait",
                                  "screen_mma_acc_wait", "screen_epi_meta_wait", "screen_epi_acc_wait",
                                  "screen_epi_test", "screen_epi_emit", "screen_epi_reserve")]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


class BatchJoin(C.Structure):
    _fields_ = [("R", C.c_void_p), ("S", C.c_void_p), ("nR", C.c_int64), ("nS", C.c_int64),
                ("d", C.c_int32), ("pad", C.c_int32), ("eps2", C.c_double)]


_lib = None


def lib() -> C.CDLL:
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise ImportError(f"{LIB_PATH} is missing: build it with tensorjoin_variants_b200._build.build() "
                          "(there is no CPU fallback)")
    L = C.CDLL(str(LIB_PATH))
    P, I64, I32, D = C.c_void_p, C.c_int64, C.c_int32, C.c_double
    L.tj_join.argtypes = [P, I64, P, I64, I32, I32, D, I32, I32, C.POINTER(Options), C.POINTER(P), P]
    L.tj_result_count.argtypes = [P]
    L.tj_result_count.restype = I64
    L.tj_result_stats.argtypes = [P, C.POINTER(Stats)]
    L.tj_result_pairs.argtypes = [P, P, P, P]
    L.tj_result_keys.argtypes = [P, P, P]
    L.tj_result_neighbor_table.argtypes = [P, P, P, P]
    L.tj_result_free.argtypes = [P]
    L.tj_result_free.restype = None
    L.tj_index_build.argtypes = [P, I64, I32, I32, D, C.POINTER(P), P]
    L.tj_index_info.argtypes = [P, C.POINTER(I64), C.POINTER(I64), C.POINTER(I64)]
    L.tj_index_copy.argtypes = [P, P, P, P, P, P]
    L.tj_index_free.argtypes = [P]
    L.tj_index_free.restype = None
    L.tj_join_batched.argtypes = [C.POINTER(BatchJoin), I32, I32, C.POINTER(Options), C.POINTER(P), P]
    L.tj_batch_offsets.argtypes = [P, P]
    L.tj_batch_pairs.argtypes = [P, P, P, P]
    L.tj_last_error_string.restype = C.c_char_p
    L.tj_version.restype = C.c_int
    L.tj_device_sm_count.restype = C.c_int
    L.tj_kernel_launches.restype = C.c_int64
    L.tj_sort_keys_noalloc.argtypes = [P, P, I64, I32, P]
    L.tj_sort_keys_noalloc.restype = C.c_int
    L.tj_pool_usage.argtypes = [C.POINTER(I64), C.POINTER(I64), C.POINTER(I64)]
    L.tj_pool_usage.restype = C.c_int
    L.tj_pool_reserve.argtypes = [I64, P]
    L.tj_pool_reserve.restype = C.c_int
    L.tj_pool_trim.argtypes = [I64]
    L.tj_pool_trim.restype = C.c_int
    L.tj_set_wait_limit.argtypes = [I64]
    L.tj_set_wait_limit.restype = C.c_int
    L.tj_result_stage_keys.argtypes = [P, I32, P, C.POINTER(I64), P]
    L.tj_result_stage_keys.restype = C.c_int
    for name in ("tj_join", "tj_result_stats", "tj_result_pairs", "tj_result_keys", "tj_result_neighbor_table",
                 "tj_index_build", "tj_index_info", "tj_index_copy", "tj_join_batched", "tj_batch_offsets",
                 "tj_batch_pairs"):
        getattr(L, name).restype = C.c_int
    _lib = L
    return L


def check(rc: int) -> None:
    if rc != TJ_OK:
        msg = lib().tj_last_error_string()
        raise TJError(rc, msg.decode() if msg else "")
