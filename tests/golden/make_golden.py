"""Regenerate the golden fixtures of tests/golden/.

Run from the repository root, naming the reference's small_matrices folder
when the .bmtx fixtures should be refreshed from it (the fixtures are
committed, so tests never need the reference tree):

    python tests/golden/make_golden.py [--bmtx-dir <reference>/small_matrices]

What it writes:
  * n16_full.bmtx, n1024.bmtx — the reference's own small_matrices fixtures
    (data files, copied byte for byte);
  * kat_bitmask.json — the known answers of the reference's bitmask test
    (test/test_compression.cu:106-238 and :550-590), restated by hand from the
    code: inputs and the outputs the reference functions produce with the
    production MASK_SIZE = 8 (include/common.h:63-65);
  * oracle_bmtx.json — digests of the oracle's A·A for the two fixtures, which
    pin the oracle's structure (and value sums) across machines.
"""
import argparse
import hashlib
import json
import os
import shutil
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))


def kats():
    return {
        "source": "test/test_compression.cu:550-590 (gen_bitmask, intersect_bitmasks) and :106-238 (tmp_test1)",
        "mask_size": 8,
        "gen_bitmask": [
            {"ptr": [0, 0, 1, 1, 3, 3, 6, 6], "mask": [0x2A]},
            {"ptr": [0, 1, 2, 2, 3, 4, 4, 5, 6], "mask": [0xDB]},
            {"ptr": [0, 0, 1, 2, 2, 3, 4, 4, 5], "mask": [0xB6]},
        ],
        "intersect_bitmasks": [{"a": [0xDB], "b": [0xB6], "out": [0x92]}],
        "tmp_test1": {
            "val": [float(x) for x in range(1, 28)],
            "col": [0, 1, 3, 7, 0, 1, 4, 7, 8, 10, 0, 2, 4, 6, 8, 1, 3, 5, 7, 9, 2, 8, 1, 5, 7, 0, 10],
            "ptr": [0, 1, 4, 10, 15, 20, 22, 25, 27],
            "mask": [3, 9],
            "expect_col": [0, 1, 3, 7],
            "expect_val": [1.0, 2.0, 3.0, 4.0],
            "expect_ptr": [0, 1, 4, 4, 4, 4, 4, 4, 4],
            "expect_nnz": 4,
            "note": ("The test comments assume MASK_SIZE=4 (rows {0,1,4,7} kept, ptr "
                     "[0,1,4,4,4,9,9,9,11]); with the production MASK_SIZE=8 only byte 0 "
                     "covers the 8 rows and bits 0,1 keep rows {0,1}."),
        },
    }


def digest(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--bmtx-dir", default=None,
                    help="the reference's small_matrices folder to copy the .bmtx fixtures from")
    args = ap.parse_args()
    if args.bmtx_dir:
        for f in ("n16_full.bmtx", "n1024.bmtx"):
            shutil.copyfile(os.path.join(args.bmtx_dir, f), os.path.join(HERE, f))
    with open(os.path.join(HERE, "kat_bitmask.json"), "w") as fh:
        json.dump(kats(), fh, indent=1)
    sys.path.insert(0, ROOT)
    import oracle
    from trident_b200 import workloads
    out = {}
    for f in ("n16_full.bmtx", "n1024.bmtx"):
        A = workloads.read_bmtx(os.path.join(HERE, f))
        rp, cj, cx, ca = oracle.spgemm(A, A)
        out[f] = {"nrows": A.nrows, "nnz_A": A.nnz, "nnz_C": int(rp[-1]), "rowptr_sha256": digest(rp),
                  "col_sha256": digest(cj), "val_sum": float(np.sum(cx)), "abs_sum": float(np.sum(ca))}
    with open(os.path.join(HERE, "oracle_bmtx.json"), "w") as fh:
        json.dump(out, fh, indent=1)
    print(json.dumps(out, indent=1))


if __name__ == "__main__":
    main()
