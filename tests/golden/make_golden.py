"""Generate the golden fixtures under tests/golden/ (run where the reference tree is available).

Usage: python tests/golden/make_golden.py --reference <path of the tensorjoin-variants checkout>
(or set TJ_REFERENCE_ROOT).  The fixture is read from
<reference>/tensorjoin_20260902_certified_exact_join/adapters/gds_g2a/test_dat.txt.

1. ``gds_test_dat_f32.npy``: GDS-Join's shipped 2-D test set
   (tensorjoin_20260902_certified_exact_join/adapters/gds_g2a/test_dat.txt,
   100,000 points, MIT licence) parsed to FP32 exactly as GDS does with
   DTYPE=float (``std::stringstream >> float``, i.e. correctly rounded
   decimal -> binary32, via C ``strtof``).  GDS's README
   (adapters/gds_g2a/README.md:80-84) states that this file at eps=1.0 in single
   precision yields 27,982,028 neighbours (directed pairs incl. self pairs).
2. ``golden.json``: counts and SHA-256 hashes of the oracle's canonical key
   arrays for the fixture and for small seeded cases, so the oracle can be
   pinned on a host without the reference tree.
"""
from __future__ import annotations

import argparse
import ctypes
import hashlib
import json
import os
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
PROJECT = "tensorjoin_20260902_certified_exact_join"


def parse_gds(path: Path) -> np.ndarray:
    libc = ctypes.CDLL("libc.so.6")
    libc.strtof.restype = ctypes.c_float
    libc.strtof.argtypes = [ctypes.c_char_p, ctypes.c_void_p]
    rows = []
    for line in path.read_text().splitlines():
        if line.strip():
            rows.append([libc.strtof(tok.strip().encode(), None) for tok in line.split(",")])
    return np.array(rows, dtype=np.float32)


def sha(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a, dtype="<u8").tobytes()).hexdigest()


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=os.environ.get("TJ_REFERENCE_ROOT"),
                    help="root of the reference checkout (or TJ_REFERENCE_ROOT)")
    args = ap.parse_args()
    if not args.reference:
        ap.error("give --reference or set TJ_REFERENCE_ROOT")
    ref = Path(args.reference) / PROJECT
    sys.path.insert(0, str(ROOT))
    import oracle
    from tensorjoin_variants_b200 import workloads as W

    X = parse_gds(ref / "adapters/gds_g2a/test_dat.txt")
    assert X.shape == (100_000, 2)
    np.save(HERE / "gds_test_dat_f32.npy", X)
    directed = oracle.join_f32(X, None, 1.0, "directed")
    upper = oracle.join_f32(X, None, 1.0, "upper")
    # GDS's own single-precision predicate: float running sum (FMA-contracted) and sqrt(d) <= eps.
    near = oracle.join_f32(X, None, 1.0 + 1e-4, "upper")
    ni, nj = oracle.keys_to_ij(near, len(X))
    a = (X[ni, 0] - X[nj, 0]).astype(np.float32)
    b = (X[ni, 1] - X[nj, 1]).astype(np.float32)
    d32 = (a.astype(np.float64) * a + b.astype(np.float64) * b).astype(np.float32)
    in32 = int(np.count_nonzero(np.sqrt(d32) <= np.float32(1.0)))
    in64 = int(np.count_nonzero(oracle.pair_d2(X, X, ni, nj) <= 1.0))
    gds_fp32_directed = len(directed) + 2 * (in32 - in64)
    golden = {
        "gds_test_dat": {
            "source": "adapters/gds_g2a/test_dat.txt", "eps": 1.0, "T": 1.0,
            "gds_readme_neighbours": 27982028,
            "gds_fp32_emulated_directed": int(gds_fp32_directed),
            "oracle_directed_count": int(len(directed)), "oracle_directed_sha256": sha(directed),
            "oracle_upper_count": int(len(upper)), "oracle_upper_sha256": sha(upper),
        }
    }
    w = W.uniform16()
    k = oracle.join_f32(w.R, None, w.T, "upper")
    golden["uniform16"] = {"eps": w.eps, "T": w.T, "oracle_upper_count": int(len(k)), "oracle_upper_sha256": sha(k),
                           "scipy_upper_equal": bool(np.array_equal(k, oracle.scipy_join(w.R, None, w.T, "upper")))}
    (HERE / "golden.json").write_text(json.dumps(golden, indent=2) + "\n")
    print(json.dumps(golden, indent=2))


if __name__ == "__main__":
    main()
