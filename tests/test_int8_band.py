"""Why the FP32-data path has no INT8 screen: the band it would certify, measured on config-2 data.

The reference's fastest FP32 pipeline quantises every vector to INT8 with its own scale
(s = max|x| / 127, q = rint(x / s); tensorjoin_20260902_certified_exact_join/src/run_d1_triton.py:82-90)
and certifies a pair from the quantised distance and the per-vector residuals e = |x - q s|:
|(|x - y|) - |q_x s_x - q_y s_y|| <= e_x + e_y (src/run_d1_triton.py:110-203,
src/g4b_r1_ragged_safe_kernel.py:8-123).  Every pair whose quantised distance lies within
e_x + e_y of eps must be refined in FP64.  This library's BF16 hi/lo screen certifies in squared
distance with the radius R = g |z||w| + c0 + |x - z||y| + |z||y - w| + |z_lo||w_lo| on centred rows
(its kernels' certificate), whose residual terms are ~2^-16 of the row norms instead of ~2^-8.

Both bounds are evaluated here on seeded config-2 rows (64-d Gaussian mixture, std 0.05,
eps for ~16 neighbours; 300 R rows x 40,000 S rows), on the same pairs, and the number of pairs
each leaves undecided is compared: the INT8 band is ~50x wider than the BF16 hi/lo band and ~4x the
result itself.  At config 2's full size the BF16 hi/lo band is 2.2M pairs, so an INT8 screen would
send ~10^8 pairs (~60 GB of gathered rows) to the FP64 refinement, more time than the whole BF16
hi/lo join takes, while the screen epilogue (not the MMA) bounds the screen at d = 64 either way.
CPU only (NumPy; the two certificates restated).
"""
import math

import numpy as np
import torch

from tensorjoin_variants_b200 import workloads as W


def _bf16(x: np.ndarray) -> np.ndarray:
    return torch.from_numpy(np.ascontiguousarray(x, dtype=np.float32)).bfloat16().float().numpy().astype(np.float64)


def _bands(n=40_000, rows=300, seed=2):
    w = W.mixture64(n=n, samples=1 << 18, seed=seed)
    R = w.R[:rows].astype(np.float64)
    S = w.S.astype(np.float64)
    T = float(w.T)
    eps = math.sqrt(T)
    D = ((R[:, None, :] - S[None, :, :]) ** 2).sum(-1)             # FP64 squared distances
    # INT8 per-vector quantisation and its distance-space interval
    def quant(X):
        s = np.abs(X).max(1, keepdims=True) / 127.0
        s[s == 0] = 1.0
        Z = np.clip(np.rint(X / s), -127, 127) * s
        return Z, np.sqrt(((X - Z) ** 2).sum(1))
    Zr, er = quant(R)
    Zs, es = quant(S)
    dq = np.sqrt(np.maximum(((Zr[:, None, :] - Zs[None, :, :]) ** 2).sum(-1), 0.0))
    wid = er[:, None] + es[None, :]
    band8 = (dq - wid <= eps) & (dq + wid > eps)
    # BF16 hi/lo screen on rows centred by the mean of both sides
    c = np.concatenate([w.R, w.S]).astype(np.float64).mean(0).astype(np.float32).astype(np.float64)
    def split(X):
        Xc = X - c
        hi = _bf16(Xc)
        lo = _bf16(Xc - hi)
        Z = hi + lo
        return (np.sqrt((Xc ** 2).sum(1)), np.sqrt((Z ** 2).sum(1)), np.sqrt(((Xc - Z) ** 2).sum(1)),
                np.sqrt((lo ** 2).sum(1)))
    yr, zr, fr, lr = split(R)
    ys, zs, fs, ls = split(S)
    K = 3 * 64
    g = (K + 64) * 2.0 ** -22
    rad = g * zr[:, None] * zs[None, :] + fr[:, None] * ys[None, :] + zr[:, None] * fs[None, :] + \
        lr[:, None] * ls[None, :]
    band3 = np.abs(D - T) <= 2.0 * rad
    return int(band8.sum()), int(band3.sum()), int((D <= T).sum()), D.size


def test_int8_band_is_far_wider_than_bf16x3_on_config2():
    b8, b3, true_pairs, pairs = _bands()
    print(f"config-2 sample: {pairs} pairs, {true_pairs} within eps; INT8 per-vector band {b8} "
          f"({b8 / pairs:.2e} of pairs), BF16 hi/lo band {b3} ({b3 / pairs:.2e})")
    assert true_pairs > 0
    assert b8 > 20 * max(b3, 1)    # measured here: 23,613 vs 455 (52x)
    assert b8 > 3 * true_pairs     # the INT8 band is several times the result itself (4.3x)
