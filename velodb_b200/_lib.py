"""Loader for ``libvelo_obl.so`` (the C ABI of include/velo_obl.h).

The library is the product: there is no Python or CPU fallback.  If it is not
built, every entry point raises instead of computing anything.
"""
from __future__ import annotations

import ctypes as C
import os

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "libvelo_obl.so")

vp, sz, u32, u64, i32, i64, u8 = C.c_void_p, C.c_size_t, C.c_uint32, C.c_uint64, C.c_int32, C.c_int64, C.c_uint8

# name -> (restype, argtypes); every function of include/velo_obl.h
PROTOS = {
    "velo_next_pow2": (sz, [sz]),
    "velo_last_error_text": (C.c_char_p, []),
    "velo_set_stage_timing": (None, [i32]),
    "velo_set_pass_timing": (None, [i32]),
    "velo_set_merge_pipeline": (None, [i32]),
    "velo_set_tensor_tile_loads": (None, [i32]),
    "velo_tensor_tile_status": (i32, []),
    "velo_pass_times_clear": (None, []),
    "velo_last_pass_times": (i32, [vp, i32]),
    "velo_trace_enabled": (i32, []),
    "velo_trace_begin": (i32, [u64, u64]),
    "velo_trace_end": (i32, [vp, vp, vp, u64, vp]),
    "velo_widen_i64": (i32, [vp, u32, sz, vp, vp]),
    "velo_ogroupby_scratch_bytes": (sz, [sz]),
    "velo_ogroupby": (i32, [vp, u32, vp, u32, u32, vp, sz, sz, vp, vp, vp, vp, vp, sz, vp]),
    "velo_device_alloc": (i32, [sz, vp, vp]),
    "velo_device_free": (i32, [vp, vp]),
    "velo_copy": (i32, [vp, vp, sz, u32, vp]),
    "velo_memset": (i32, [vp, i32, sz, vp]),
    "velo_stream_sync": (i32, [vp]),
    "velo_range_mask": (i32, [vp, u32, sz, i64, i64, vp, u32, vp]),
    "velo_iota_i64": (i32, [vp, sz, i64, vp]),
    "velo_ocompact_columns_scratch_bytes": (sz, [sz]),
    "velo_ocompact_columns": (i32, [vp, vp, vp, u32, vp, sz, vp, vp, sz, vp]),
    "velo_ogather_column_scratch_bytes": (sz, [sz, sz]),
    "velo_ogather_column": (i32, [vp, u32, vp, sz, vp, sz, vp, vp, vp, sz, vp]),
    "velo_last_stage_times": (i32, [vp, i32]),
    "velo_osort_kp": (i32, [vp, vp, sz, sz, vp, vp]),
    "velo_sort_columns": (i32, [vp, vp, vp, u32, sz, sz, vp, vp, sz, vp]),
    "velo_sort_scratch_bytes": (sz, [vp, u32, sz]),
    "velo_osort_records": (i32, [vp, u32, u64, sz, sz, u32, vp, vp]),
    "velo_ocompact_kpm": (i32, [vp, vp, vp, sz, sz, vp, vp, sz, vp, vp]),
    "velo_compact_scratch_bytes": (sz, [sz, vp]),
    "velo_ocompact_kpm_noalloc": (i32, [vp, vp, vp, sz, sz, vp, vp]),
    "velo_permute": (i32, [vp, vp, vp, sz, u32, vp]),
    "velo_scatter_scratch_bytes": (sz, [sz]),
    "velo_scatter": (i32, [vp, sz, vp, vp, vp, sz, vp]),
    "velo_gather": (i32, [vp, vp, vp, vp, sz, u32, vp]),
    "velo_compare_eq": (i32, [vp, vp, vp, sz, u32, vp]),
    "velo_compose_position_map": (i32, [vp, vp, vp, sz, vp]),
    "velo_enrich_positions": (i32, [vp, vp, vp, sz, vp]),
    "velo_oshuffle_scratch_bytes": (sz, [sz]),
    "velo_oshuffle_position_map": (i32, [vp, sz, u64, u64, vp, sz, vp]),
    "velo_ogather_scratch_bytes": (sz, [sz, sz]),
    "velo_ogather_u64": (i32, [vp, sz, vp, sz, vp, vp, sz, vp]),
    "velo_ojoin_scratch_bytes": (sz, [sz, sz]),
    "velo_ojoin_pkfk": (i32, [vp, vp, sz, vp, vp, sz, u32, vp, vp, vp, vp, sz, vp]),
    "velo_ojoin_mn_scratch_bytes": (sz, [sz, sz, sz]),
    "velo_ojoin_mn": (i32, [vp, vp, sz, vp, vp, sz, u32, sz, vp, vp, vp, vp, sz, vp]),
    "velo_ohash_join_scratch_bytes": (sz, [sz, sz]),
    "velo_ohash_join": (i32, [vp, vp, sz, vp, vp, sz, u32, u64, vp, vp, vp, vp, sz, vp]),
    "velo_init": (i32, [vp, vp]),
    "velo_shutdown": (i32, [vp, u32]),
    "velo_submit": (i32, [vp, vp, vp]),
    "velo_batch_submit": (i32, [vp, vp, sz, vp]),
    "velo_wait": (i32, [vp, u64, u64]),
    "velo_last_error": (i32, [vp, vp, sz]),
    "velo_ctx_stream": (vp, [vp]),
    "velo_cmd_size": (sz, []),
    "velo_ctx_launches": (u64, [vp]),
    "velo_server_create": (i32, [vp, vp, vp]),
    "velo_server_submit": (i32, [vp, vp, vp]),
    "velo_server_wait": (i32, [vp, u64, u64, vp]),
    "velo_server_stats": (i32, [vp, vp]),
    "velo_server_destroy": (i32, [vp, u32]),
    "velo_batch_create": (i32, [vp, sz, vp, vp]),
    "velo_batch_launch": (i32, [vp, vp]),
    "velo_batch_status": (i32, [vp, vp]),
    "velo_batch_destroy": (None, [vp]),
    "velo_batch_set_timeout": (i32, [vp, u64]),
    "velo_batch_inject_unmet_wait": (i32, [vp, u32]),
    "velo_batch_autotune": (i32, [vp, sz, u32, vp, vp, vp]),
    "velo_filter_groupby_scratch_bytes": (sz, [sz, u32]),
    "velo_filter_groupby": (i32, [vp, sz, vp, u32, u32, vp, vp, vp, sz, vp]),
    "velo_join_groupby_topk_scratch_bytes": (sz, [sz, sz]),
    "velo_join_groupby_topk": (i32, [vp, vp, u32, vp, vp, vp, sz, vp]),
}

STATUS = {0: "VELO_OK", -1: "VELO_EINVAL", -2: "VELO_ENOMEM", -3: "VELO_ECUDA", -4: "VELO_ETIMEDOUT",
          -5: "VELO_EOVERFLOW", -6: "VELO_ESTATE", -7: "VELO_ENOTSUP"}


class VeloError(RuntimeError):
    def __init__(self, status: int, what: str, text: str):
        super().__init__(f"{what}: {STATUS.get(status, status)}: {text}")
        self.status = status


_lib = None


class VeloTune(C.Structure):
    _fields_ = [("tile_log2", C.c_uint32), ("threads", C.c_uint32)]


def lib() -> C.CDLL:
    """The loaded library; raises if it was not built (no fallback)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m velodb_b200.build`")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in PROTOS.items():
            if hasattr(L, name):
                f = getattr(L, name)
                f.restype = res
                f.argtypes = args
        _lib = L
    return _lib


def last_error() -> str:
    t = lib().velo_last_error_text()
    return t.decode() if t else ""


def check(status: int, what: str) -> None:
    if status != 0:
        raise VeloError(status, what, last_error())


class VeloPassTime(C.Structure):
    _fields_ = [("kind", C.c_uint32), ("log_n", C.c_uint32), ("row_bytes", C.c_uint32), ("ms", C.c_float)]


class VeloLineitem(C.Structure):
    _fields_ = [(n, C.c_void_p) for n in ("qty", "price", "disc", "tax", "shipdate", "flag1", "flag2")]


class VeloLineitemPred(C.Structure):
    _fields_ = [(n, C.c_int32) for n in ("ship_lo", "ship_hi", "disc_lo", "disc_hi", "qty_lo", "qty_hi")]


class VeloJoinTables(C.Structure):
    _fields_ = [("dim_key", C.c_void_p), ("dim_date", C.c_void_p), ("n_dim", C.c_size_t),
                ("fact_fk", C.c_void_p), ("fact_price", C.c_void_p), ("n_fact", C.c_size_t)]


class VeloJoinPred(C.Structure):
    _fields_ = [("date_hi", C.c_int32), ("pad_", C.c_int32), ("price_hi", C.c_int64)]


class VeloBatchItem(C.Structure):
    _fields_ = [("kind", C.c_uint32), ("pad_", C.c_uint32), ("d_keys", C.c_void_p), ("d_payload", C.c_void_p),
                ("d_marks", C.c_void_p), ("n", C.c_size_t), ("capacity", C.c_size_t), ("d_count", C.c_void_p)]


def _args(*fields):
    return type("Args", (C.Structure,), {"_fields_": [(f"f{i}", t) for i, t in enumerate(fields)]})


class VeloCmdArgs(C.Union):
    _fields_ = [
        ("permute", _args(vp, vp, vp, sz, u32)),
        ("compare_eq", _args(vp, vp, vp, sz, u32)),
        ("osort_kp", _args(vp, vp, sz, sz)),
        ("ocompact_kpm", _args(vp, vp, vp, sz, sz, vp, vp, sz)),
        ("ogather", _args(vp, sz, vp, sz, vp, vp, sz)),
        ("ojoin", _args(vp, vp, sz, vp, vp, sz, u32, vp, vp, vp, vp, sz)),
        ("ojoin_mn", _args(vp, vp, sz, vp, vp, sz, u32, sz, vp, vp, vp, vp, sz)),
        ("ohash", _args(vp, vp, sz, vp, vp, sz, u32, u64, vp, vp, vp, vp, sz)),
        ("scatter", _args(vp, sz, vp, vp, vp, sz)),
        ("gather", _args(vp, vp, vp, vp, sz, u32)),
        ("compose", _args(vp, vp, vp, sz)),
        ("enrich", _args(vp, vp, vp, sz)),
        ("oshuffle", _args(vp, sz, u64, u64, vp, sz)),
        ("filter_groupby", _args(vp, sz, vp, u32, vp, vp, vp, sz)),
        ("join_topk", _args(vp, vp, u32, vp, vp, vp, sz)),
    ]


class VeloCmd(C.Structure):
    _fields_ = [("opcode", C.c_uint32), ("flags", C.c_uint32), ("args", VeloCmdArgs)]


class VeloConfig(C.Structure):
    _fields_ = [("device", C.c_int32), ("queue_capacity", C.c_uint32), ("flags", C.c_uint32),
                ("idle_us", C.c_uint32)]


OP = dict(NOP=0, SCATTER=1, GATHER=2, SORT=3, PERMUTE=4, COMPARE_EQ=10, COMPOSE_POSITION_MAP=11, ENRICH_POSITIONS=12,
          OSORT_KP=0x100, OCOMPACT_KPM=0x101, OSORT_RECORDS=0x102, OJOIN_PKFK=0x103, OGATHER=0x104, OSHUFFLE=0x105,
          FILTER_GROUPBY=0x106, JOIN_GROUPBY_TOPK=0x107, OJOIN_MN=0x108, OHASH_JOIN=0x109)


class VeloServedTables(C.Structure):
    _fields_ = [("fact", VeloLineitem), ("fact_fk", vp), ("fact_fk32", vp), ("fact_n", sz), ("dim_key", vp),
                ("dim_key32", vp), ("dim_date", vp), ("dim_n", sz), ("fact2_fk", vp), ("fact2_price", vp),
                ("fact2_n", sz)]


class VeloQuery(C.Structure):
    _fields_ = [("shape", C.c_uint32), ("pad_", C.c_uint32), ("offset", sz), ("n", sz), ("dim_offset", sz),
                ("dim_n", sz), ("f2_offset", sz), ("f2_n", sz), ("pred", VeloLineitemPred), ("jpred", VeloJoinPred)]


class VeloQueryResult(C.Structure):
    _fields_ = [("qid", C.c_uint64), ("status", C.c_int32), ("shape", C.c_uint32), ("submit_ms", C.c_double),
                ("start_ms", C.c_double), ("end_ms", C.c_double), ("out", C.c_int64 * 96),
                ("counts", C.c_uint64 * 2)]


class VeloServerConfig(C.Structure):
    _fields_ = [("device", C.c_int32), ("slots", C.c_uint32), ("hbm_budget_bytes", C.c_uint64),
                ("flags", C.c_uint32), ("idle_us", C.c_uint32)]


class VeloServerStats(C.Structure):
    _fields_ = [(n, C.c_uint64) for n in ("admitted", "completed", "pending", "peak_inflight", "arena_bytes",
                                          "peak_arena_bytes")]


def tune_ref(tune):
    """ctypes pointer for an optional (tile_log2, threads) tuple."""
    if tune is None:
        return None
    t = VeloTune(int(tune[0]), int(tune[1]))
    return C.byref(t)
