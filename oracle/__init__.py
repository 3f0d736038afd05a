"""CPU oracle for the oblivious operator path -- TEST INFRASTRUCTURE ONLY.

ctypes bindings for ``oracle/liboracle.so`` (a plain-C restatement of the
reference algorithms, see ``oracle/oracle.h``) and, where it was built, for
``oracle/_ref/liboblivious.so`` (the reference's own CPU library compiled from
its sources by ``oracle/Makefile``).

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU legs of ``bench.py``
import this module.  The product package ``velodb_b200`` never does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
REF_PATH = os.path.join(HERE, "_ref", "liboblivious.so")

# DataTypeId values (reference include/data/data_type.hpp:12-26)
BOOLEAN, TINYINT, SMALLINT, INTEGER, BIGINT, FLOAT, DOUBLE, VARCHAR, DATE = 1, 2, 3, 4, 5, 6, 7, 8, 10
NP_OF_TYPE = {
    BOOLEAN: np.uint8, TINYINT: np.int8, SMALLINT: np.int16, INTEGER: np.int32, BIGINT: np.int64,
    FLOAT: np.float32, DOUBLE: np.float64, VARCHAR: np.uint64, DATE: np.uint32,
}

_lib = None
_ref = None


def build() -> None:
    """Compile liboracle.so (and oracle/_ref when the reference tree exists)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        vp, sz, i32 = C.c_void_p, C.c_size_t, C.c_int
        L.orc_next_pow2.argtypes = [sz]
        L.orc_next_pow2.restype = sz
        L.orc_bitonic_sort_cols.argtypes = [i32, vp, vp, vp, sz, sz, vp]
        L.orc_bitonic_sort_cols.restype = i32
        L.orc_bitonic_kp.argtypes = [vp, vp, sz, sz, i32]
        L.orc_bitonic_kp.restype = None
        L.orc_bitonic_records.argtypes = [vp, i32, i32, vp, vp, sz, sz, i32]
        L.orc_bitonic_records.restype = None
        L.orc_ocompact.argtypes = [vp, sz, sz, vp]
        L.orc_ocompact.restype = sz
        L.orc_scatter_stable.argtypes = [vp, sz, vp]
        L.orc_scatter_stable.restype = sz
        L.orc_groupby_sorted.argtypes = [vp, vp, sz, i32, vp, vp]
        L.orc_groupby_sorted.restype = sz
        L.orc_filter_groupby.argtypes = [sz] + [vp] * 7 + [C.c_int32] * 6 + [sz, vp, vp, i32]
        L.orc_filter_groupby.restype = sz
        L.orc_join_groupby_topk.argtypes = [sz, vp, vp, sz, vp, vp, C.c_int32, C.c_int64, sz, vp, vp, vp, i32]
        L.orc_join_groupby_topk.restype = sz
        u64 = C.c_uint64
        L.orc_smj_pairs.argtypes = [vp, vp, sz, vp, vp, sz, vp, vp, sz]
        L.orc_smj_pairs.restype = sz
        L.orc_obl_sort_rec2.argtypes = [vp, sz, u64, u64, i32]
        L.orc_obl_sort_rec2.restype = None
        L.orc_obl_compact_rec2.argtypes = [vp, sz, i32, i32, i32, i32]
        L.orc_obl_compact_rec2.restype = sz
        L.orc_obl_filter_groupby.argtypes = L.orc_filter_groupby.argtypes
        L.orc_obl_filter_groupby.restype = sz
        L.orc_obl_join_groupby_topk.argtypes = L.orc_join_groupby_topk.argtypes
        L.orc_obl_join_groupby_topk.restype = sz
        _lib = L
    return _lib


def ref_lib():
    """liboblivious built from the reference sources, or None when absent."""
    global _ref
    if _ref is None and os.path.exists(REF_PATH):
        R = C.CDLL(REF_PATH)
        R.o_compact.argtypes = [C.c_void_p, C.c_size_t, C.c_size_t, C.c_void_p, C.c_void_p]
        R.o_compact.restype = None
        R.o_sort.argtypes = [C.c_void_p, C.c_size_t, C.c_size_t, C.c_void_p, C.c_void_p]
        R.o_sort.restype = None
        _ref = R
    return _ref


def _p(a: np.ndarray) -> int:
    assert a.flags["C_CONTIGUOUS"]
    return a.ctypes.data


def next_pow2(x: int) -> int:
    return int(lib().orc_next_pow2(x))


# --------------------------------------------------------------------------
# sorts
# --------------------------------------------------------------------------

def bitonic_sort_cols(cols, types, ascending, n):
    """Reference OP_SORT semantics on copies of ``cols`` (each padded to
    next_pow2(n) in place).  Returns (sorted cols list, int64 indices)."""
    npad = next_pow2(n) if n > 0 else 0
    outs = []
    for c, t in zip(cols, types):
        a = np.zeros(max(npad, 1), dtype=NP_OF_TYPE[t])
        a[:n] = np.asarray(c, dtype=NP_OF_TYPE[t])[:n]
        outs.append(a)
    idx = np.zeros(max(npad, 1), dtype=np.int64)
    if n == 0:
        return [o[:0] for o in outs], idx[:0]
    ptrs = (C.c_void_p * len(outs))(*[_p(o) for o in outs])
    tarr = np.asarray(types, dtype=np.int32)
    aarr = np.asarray([1 if a else 0 for a in ascending], dtype=np.uint8)
    rc = lib().orc_bitonic_sort_cols(len(outs), C.cast(ptrs, C.c_void_p), _p(tarr), _p(aarr), n, npad, _p(idx))
    assert rc == 0
    return outs, idx


def bitonic_kp(keys, pay, n_threads=0):
    """(u64 key, u32 payload) network sort; returns padded arrays."""
    n = len(keys)
    npad = next_pow2(n)
    k = np.empty(npad, np.uint64)
    p = np.empty(npad, np.uint32)
    k[:n] = keys
    p[:n] = pay
    lib().orc_bitonic_kp(_p(k), _p(p), n, npad, n_threads)
    return k, p


def bitonic_records(words, n_key_words, masks, pad, n_threads=0):
    """Record network sort over SoA u64 words; returns padded word arrays."""
    n = len(words[0])
    npad = next_pow2(n)
    ws = []
    for w in words:
        a = np.empty(npad, np.uint64)
        a[:n] = w
        ws.append(a)
    ptrs = (C.c_void_p * len(ws))(*[_p(w) for w in ws])
    m = np.asarray(masks, dtype=np.uint64)
    pd = np.asarray(pad, dtype=np.uint64)
    lib().orc_bitonic_records(C.cast(ptrs, C.c_void_p), len(ws), n_key_words, _p(m), _p(pd), n, npad, n_threads)
    return ws


# --------------------------------------------------------------------------
# compaction
# --------------------------------------------------------------------------

def ocompact(data: np.ndarray, marks: np.ndarray):
    """ORCompact restatement over the rows of a 2-D uint8 (or any) array.
    Returns (compacted data, compacted marks, count)."""
    d = np.ascontiguousarray(data).copy()
    m = np.ascontiguousarray(marks.astype(np.uint8)).copy()
    n = d.shape[0]
    esz = d.nbytes // n if n else 1
    cnt = lib().orc_ocompact(_p(d), n, esz, _p(m)) if n else 0
    return d, m, int(cnt)


_IS_MARKED = C.CFUNCTYPE(C.c_bool, C.c_void_p, C.c_void_p)


def ref_o_compact(values: np.ndarray, marks: np.ndarray):
    """Reference liboblivious o_compact over (u64 value, u64 mark) elements.
    Returns (values, marks) after compaction, or None when not built."""
    R = ref_lib()
    if R is None:
        return None
    n = len(values)
    el = np.empty((n, 2), dtype=np.uint64)
    el[:, 0] = values
    el[:, 1] = marks.astype(np.uint64)

    def is_marked(ptr, aux):
        return C.cast(ptr, C.POINTER(C.c_uint64))[1] != 0

    cb = _IS_MARKED(is_marked)
    R.o_compact(_p(el), n, 16, C.cast(cb, C.c_void_p), None)
    return el[:, 0].copy(), el[:, 1].copy()


_CMP = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_void_p, C.c_void_p)


def ref_o_sort_u64(values: np.ndarray):
    """Reference liboblivious o_sort (Batcher odd-even merge) over u64s."""
    R = ref_lib()
    if R is None:
        return None
    a = np.ascontiguousarray(values, dtype=np.uint64).copy()

    def cmp(pa, pb, aux):
        x = C.cast(pa, C.POINTER(C.c_uint64))[0]
        y = C.cast(pb, C.POINTER(C.c_uint64))[0]
        return (x > y) - (x < y)

    cb = _CMP(cmp)
    R.o_sort(_p(a), len(a), 8, C.cast(cb, C.c_void_p), None)
    return a


def scatter_stable(mask: np.ndarray):
    m = np.ascontiguousarray(mask.astype(np.uint8))
    idx = np.full(len(m), -1, dtype=np.int32)
    cnt = lib().orc_scatter_stable(_p(m), len(m), _p(idx)) if len(m) else 0
    return idx, int(cnt)


# --------------------------------------------------------------------------
# group-by and pipelines
# --------------------------------------------------------------------------

def groupby_sorted(keys: np.ndarray, vals: np.ndarray):
    keys = np.ascontiguousarray(keys, dtype=np.uint64)
    vals = np.ascontiguousarray(vals, dtype=np.int64)
    n, v = vals.shape
    ok = np.empty(max(n, 1), np.uint64)
    os_ = np.empty((max(n, 1), v), np.int64)
    g = lib().orc_groupby_sorted(_p(keys), _p(vals), n, v, _p(ok), _p(os_)) if n else 0
    return ok[:g], os_[:g]


def filter_groupby(cols: dict, pred: dict, max_groups: int = 8, n_threads: int = 0, oblivious: bool = False):
    """Filter + group-by oracle.  cols: qty, price, disc, tax, shipdate, flag1,
    flag2 (numpy arrays); pred: ship_lo/ship_hi/disc_lo/disc_hi/qty_lo/qty_hi.
    Returns (group count, keys[g], sums[g, 5]).  oblivious=True runs the
    oblivious CPU pipeline (orc_obl_filter_groupby: ORCompact and a network
    sort over all next_pow2(n) rows) instead of the count-revealing one."""
    n = len(cols["qty"])
    arrs = [np.ascontiguousarray(cols[k]) for k in ("qty", "price", "disc", "tax", "shipdate", "flag1", "flag2")]
    ok = np.zeros(max_groups, np.uint64)
    os_ = np.zeros((max_groups, 5), np.int64)
    fn = lib().orc_obl_filter_groupby if oblivious else lib().orc_filter_groupby
    g = fn(n, *[_p(a) for a in arrs], pred["ship_lo"], pred["ship_hi"], pred["disc_lo"], pred["disc_hi"],
           pred["qty_lo"], pred["qty_hi"], max_groups, _p(ok), _p(os_), n_threads)
    g = int(g)
    return g, ok[:min(g, max_groups)], os_[:min(g, max_groups)]


def join_groupby_topk(dim: dict, fact: dict, pred: dict, k: int = 10, n_threads: int = 0, oblivious: bool = False):
    """PK-FK join + group-by + top-k oracle; returns (n_groups, fk, sum, cnt).
    oblivious=True runs the oblivious CPU pipeline (orc_obl_join_groupby_topk)."""
    dk = np.ascontiguousarray(dim["key"], np.int32)
    dd = np.ascontiguousarray(dim["date"], np.int32)
    ff = np.ascontiguousarray(fact["fk"], np.int32)
    fp = np.ascontiguousarray(fact["price"], np.int64)
    ofk = np.zeros(k, np.int32)
    osum = np.zeros(k, np.int64)
    ocnt = np.zeros(k, np.int64)
    fn = lib().orc_obl_join_groupby_topk if oblivious else lib().orc_join_groupby_topk
    g = fn(len(dk), _p(dk), _p(dd), len(ff), _p(ff), _p(fp), pred["date_hi"], pred["price_hi"], k, _p(ofk),
           _p(osum), _p(ocnt), n_threads)
    g = int(g)
    m = min(g, k)
    return g, ofk[:m], osum[:m], ocnt[:m]


def smj_pairs(left_keys, left_mask, right_keys, right_mask, cap=None):
    """Reference sort-merge join output: (left row ids, right row ids,
    total pairs) in (key, left row id, right row id) order."""
    lk = np.ascontiguousarray(left_keys, dtype=np.int64)
    rk = np.ascontiguousarray(right_keys, dtype=np.int64)
    lm = None if left_mask is None else np.ascontiguousarray(left_mask, dtype=np.uint8)
    rm = None if right_mask is None else np.ascontiguousarray(right_mask, dtype=np.uint8)
    if cap is None:
        cap = lib().orc_smj_pairs(_p(lk), None if lm is None else _p(lm), len(lk), _p(rk),
                                  None if rm is None else _p(rm), len(rk), None, None, 0)
    ol = np.zeros(max(int(cap), 1), np.int64)
    orr = np.zeros(max(int(cap), 1), np.int64)
    tot = lib().orc_smj_pairs(_p(lk), None if lm is None else _p(lm), len(lk), _p(rk),
                              None if rm is None else _p(rm), len(rk), _p(ol), _p(orr), int(cap))
    m = min(int(tot), int(cap))
    return ol[:m], orr[:m], int(tot)


def obl_sort_rec2(recs: np.ndarray, m0: int, m1: int, n_threads: int = 0) -> np.ndarray:
    """Oblivious CPU network sort of (n, 2) u64 records (n a power of two)."""
    r = np.ascontiguousarray(recs, dtype=np.uint64).copy()
    lib().orc_obl_sort_rec2(_p(r), r.shape[0], m0, m1, n_threads)
    return r


def obl_compact_rec2(recs: np.ndarray, word: int, bit: int, inv: int, n_threads: int = 0):
    """Oblivious CPU ORCompact of (n, 2) u64 records (n a power of two)."""
    r = np.ascontiguousarray(recs, dtype=np.uint64).copy()
    c = lib().orc_obl_compact_rec2(_p(r), r.shape[0], word, bit, inv, n_threads)
    return r, int(c)


# --------------------------------------------------------------------------
# Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as
# easy as 1, 2, 3", SC'11), restated in numpy: the keys of the device shuffle
# --------------------------------------------------------------------------

def philox_u64(idx: np.ndarray, counter: int, key: int) -> np.ndarray:
    idx = np.asarray(idx, dtype=np.uint64)
    m32 = np.uint64(0xFFFFFFFF)
    c0 = idx & m32
    c1 = idx >> np.uint64(32)
    c2 = np.full_like(idx, counter & 0xFFFFFFFF)
    c3 = np.full_like(idx, (counter >> 32) & 0xFFFFFFFF)
    k0, k1 = key & 0xFFFFFFFF, (key >> 32) & 0xFFFFFFFF
    with np.errstate(over="ignore"):
        for _ in range(10):
            p0 = np.uint64(0xD2511F53) * c0
            p1 = np.uint64(0xCD9E8D57) * c2
            hi0, lo0 = p0 >> np.uint64(32), p0 & m32
            hi1, lo1 = p1 >> np.uint64(32), p1 & m32
            c0, c1, c2, c3 = hi1 ^ c1 ^ np.uint64(k0), lo1, hi0 ^ c3 ^ np.uint64(k1), lo0
            k0 = (k0 + 0x9E3779B9) & 0xFFFFFFFF
            k1 = (k1 + 0xBB67AE85) & 0xFFFFFFFF
    return (c1 << np.uint64(32)) | c0


def shuffle_position_map(pmap: np.ndarray, key: int, counter: int) -> np.ndarray:
    """map o sigma, sigma sorting the Philox keys (ties by map value, which the
    network compares too)."""
    n = len(pmap)
    k = philox_u64(np.arange(n, dtype=np.uint64), counter, key)
    order = np.lexsort((pmap.astype(np.uint64), k))
    return pmap[order]
