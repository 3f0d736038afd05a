"""Generates the golden fixtures in this folder from the reference's own code.

Run here (where the reference tree exists):  python tests/golden/make_golden.py

* ``liboblivious_compact.npz`` -- outputs of liboblivious ``o_compact``
  (obliviator/operator_1/third_party/liboblivious/algorithms.c:116-213, built
  from the reference sources by oracle/Makefile into oracle/_ref/) on seeded
  (u64 value, mark) inputs of many sizes, power-of-two and not.
* ``liboblivious_sort.npz`` -- outputs of liboblivious ``o_sort`` (Batcher
  odd-even mergesort, algorithms.c:7-114) on seeded u64 inputs.

Inputs are regenerated from ``velodb_b200.workloads`` (splitmix64 streams), so
only the outputs are stored.  The fixtures let tests pin the oracle and the
GPU kernels on machines without the reference tree.
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from velodb_b200 import workloads as W  # noqa: E402

COMPACT_SIZES = list(range(1, 65)) + [96, 100, 127, 128, 129, 255, 256, 257, 1000, 1024, 2047, 2048, 4096, 5000,
                                      8192, 8193, 20000]
SORT_SIZES = [1, 2, 3, 7, 8, 100, 1000, 1024, 4097]
SEED = 0xB2000000000000C0


def compact_inputs(n: int, case: int):
    vals = W.splitmix64(SEED, n, 2 * case)
    # keep probability 0.3 / 0.5 / 0.9 by case, from an independent stream
    thr = [3, 5, 9][case % 3]
    marks = (W.lemire(W.splitmix64(SEED, n, 2 * case + 1), 10) < thr).astype(np.uint8)
    return vals, marks


def sort_inputs(n: int, case: int):
    return W.splitmix64(SEED ^ 0x5, n, case)


def main():
    oracle.build()
    if oracle.ref_lib() is None:
        raise SystemExit("oracle/_ref/liboblivious.so is missing (needs the reference tree)")
    # values are distinct, so each output is stored as the input position of
    # every output element (uint16), which compresses far better than values
    out_p, sizes = [], []
    for case, n in enumerate(COMPACT_SIZES):
        vals, marks = compact_inputs(n, case)
        rv, rm = oracle.ref_o_compact(vals, marks)
        pos = {int(v): i for i, v in enumerate(vals)}
        perm = np.asarray([pos[int(v)] for v in rv], dtype=np.uint16)
        assert np.array_equal(rm.astype(np.uint8), marks[perm])
        out_p.append(perm)
        sizes.append(n)
    np.savez_compressed(os.path.join(HERE, "liboblivious_compact.npz"), sizes=np.asarray(sizes, np.int64),
                        perm=np.concatenate(out_p))
    out_s, ssz = [], []
    for case, n in enumerate(SORT_SIZES):
        vals = sort_inputs(n, case)
        rv = oracle.ref_o_sort_u64(vals)
        pos = {int(v): i for i, v in enumerate(vals)}
        out_s.append(np.asarray([pos[int(v)] for v in rv], dtype=np.uint16))
        ssz.append(n)
    np.savez_compressed(os.path.join(HERE, "liboblivious_sort.npz"), sizes=np.asarray(ssz, np.int64),
                        perm=np.concatenate(out_s))
    print("wrote", os.listdir(HERE))


if __name__ == "__main__":
    main()
