"""Thin Python calls into the C ABI over torch device buffers.

torch only provides device memory and streams here; every byte of the
operators is computed by the sm_100a kernels in libvelo_obl.so.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from ._lib import check, lib, tune_ref


def _stream(stream):
    if stream is None:
        return torch.cuda.current_stream().cuda_stream
    return stream.cuda_stream if hasattr(stream, "cuda_stream") else stream


def next_pow2(x: int) -> int:
    return int(lib().velo_next_pow2(x))


def set_stage_timing(on: bool) -> None:
    """Switch the pipelines' per-stage CUDA-event timing (velo_set_stage_timing)."""
    lib().velo_set_stage_timing(1 if on else 0)


def last_stage_times() -> list:
    """Stage durations (ms) of this thread's last timed pipeline call."""
    buf = np.zeros(8, dtype=np.float32)
    n = int(lib().velo_last_stage_times(buf.ctypes.data, 8))
    return [float(x) for x in buf[:n]]


PASS_KINDS = {0: "tile_sort", 1: "merge", 2: "global", 3: "compact_tile", 4: "compact_global"}


def set_pass_timing(on: bool) -> None:
    """Switch per-pass CUDA-event timing of the network passes
    (velo_set_pass_timing); clears this thread's pass list."""
    lib().velo_set_pass_timing(1 if on else 0)


def set_merge_pipeline(on: bool) -> None:
    """Tune: in-tile merge passes as persistent CTAs with bulk-copy prefetch
    (velo_set_merge_pipeline); off by default."""
    lib().velo_set_merge_pipeline(1 if on else 0)


def set_tensor_tile_loads(on: bool) -> None:
    """Tune: merge and fused global passes load their rows with tensor-map
    tile copies (velo_set_tensor_tile_loads); off by default."""
    lib().velo_set_tensor_tile_loads(1 if on else 0)


def tensor_tile_status() -> int:
    """0 unless a tensor-map pass kernel recorded a fault code
    (velo_tensor_tile_status)."""
    return int(lib().velo_tensor_tile_status())


TUNES = {"merge_pipeline": set_merge_pipeline, "tensor_tile_loads": set_tensor_tile_loads}


def clear_pass_times() -> None:
    lib().velo_pass_times_clear()


def last_pass_times() -> list:
    """(kind name, log2 rows, row bytes, ms) of every network pass this thread
    launched since the list was last cleared."""
    from ._lib import VeloPassTime

    buf = (VeloPassTime * 1024)()
    n = int(lib().velo_last_pass_times(C.cast(buf, C.c_void_p), 1024))
    return [(PASS_KINDS.get(int(buf[i].kind), str(buf[i].kind)), int(buf[i].log_n), int(buf[i].row_bytes),
             float(buf[i].ms)) for i in range(n)]


def to_dev_u64(a: np.ndarray, capacity: int | None = None, device="cuda") -> torch.Tensor:
    """Upload a uint64 array into an int64 device tensor of `capacity` rows."""
    cap = len(a) if capacity is None else capacity
    t = torch.empty(max(cap, 1), dtype=torch.int64, device=device)
    if len(a):
        t[: len(a)].copy_(torch.from_numpy(np.ascontiguousarray(a).view(np.int64)))
    return t


def to_dev_u32(a: np.ndarray, capacity: int | None = None, device="cuda") -> torch.Tensor:
    cap = len(a) if capacity is None else capacity
    t = torch.empty(max(cap, 1), dtype=torch.int32, device=device)
    if len(a):
        t[: len(a)].copy_(torch.from_numpy(np.ascontiguousarray(a).view(np.int32)))
    return t


def to_dev_u8(a: np.ndarray, capacity: int | None = None, device="cuda") -> torch.Tensor:
    cap = len(a) if capacity is None else capacity
    t = torch.zeros(max(cap, 1), dtype=torch.uint8, device=device)
    if len(a):
        t[: len(a)].copy_(torch.from_numpy(np.ascontiguousarray(a).astype(np.uint8)))
    return t


def host_u64(t: torch.Tensor, n: int | None = None) -> np.ndarray:
    a = t.cpu().numpy().view(np.uint64)
    return a if n is None else a[:n]


def host_u32(t: torch.Tensor, n: int | None = None) -> np.ndarray:
    a = t.cpu().numpy().view(np.uint32)
    return a if n is None else a[:n]


# --------------------------------------------------------------------------

def osort_kp(keys: torch.Tensor, pay: torch.Tensor, n: int, tune=None, stream=None) -> None:
    """In-place oblivious sort of (u64 key, u32 payload) rows (velo_osort_kp)."""
    cap = min(keys.numel(), pay.numel())
    check(lib().velo_osort_kp(keys.data_ptr(), pay.data_ptr(), n, cap, tune_ref(tune), _stream(stream)),
          "velo_osort_kp")


def compact_scratch_bytes(capacity: int, tune=None) -> int:
    return int(lib().velo_compact_scratch_bytes(capacity, tune_ref(tune)))


def ocompact_kpm(keys, pay, marks, n: int, tune=None, stream=None, scratch=None) -> torch.Tensor:
    """In-place ORCompact of (key, payload, mark) rows; returns the device
    count tensor (uint64 stored in an int64 tensor)."""
    cap = min(keys.numel(), pay.numel(), marks.numel())
    nbytes = compact_scratch_bytes(cap, tune)
    if scratch is None:
        scratch = torch.empty(max(nbytes, 1), dtype=torch.uint8, device=keys.device)
    cnt = torch.zeros(1, dtype=torch.int64, device=keys.device)
    check(lib().velo_ocompact_kpm(keys.data_ptr(), pay.data_ptr(), marks.data_ptr(), n, cap, cnt.data_ptr(),
                                  scratch.data_ptr(), scratch.numel(), tune_ref(tune), _stream(stream)),
          "velo_ocompact_kpm")
    return cnt


def sort_scratch_bytes(types, n: int) -> int:
    t = np.asarray(types, dtype=np.uint32)
    return int(lib().velo_sort_scratch_bytes(t.ctypes.data, len(t), n))


def sort_columns(cols, types, ascending, n: int, stream=None):
    """Reference OP_SORT contract (velo_sort_columns): sorts the device
    columns in place over next_pow2(n) rows and returns the int64 indices."""
    t = np.asarray(types, dtype=np.uint32)
    a = np.asarray([1 if x else 0 for x in ascending], dtype=np.uint8)
    ptrs = np.asarray([c.data_ptr() for c in cols], dtype=np.uint64)
    cap = min(c.numel() * c.element_size() // _elem_size(tt) for c, tt in zip(cols, types)) if cols else 0
    dev = cols[0].device
    idx = torch.empty(max(next_pow2(n), 1), dtype=torch.int64, device=dev)
    nb = sort_scratch_bytes(types, n)
    scratch = torch.empty(max(nb, 1), dtype=torch.uint8, device=dev)
    check(lib().velo_sort_columns(ptrs.ctypes.data, t.ctypes.data, a.ctypes.data, len(cols), n, cap, idx.data_ptr(),
                                  scratch.data_ptr(), scratch.numel(), _stream(stream)), "velo_sort_columns")
    return idx


_SIZES = {1: 1, 2: 1, 3: 2, 4: 4, 5: 8, 6: 4, 7: 8, 8: 8, 10: 4}


def _elem_size(t: int) -> int:
    return _SIZES[int(t)]


REVEAL_COUNT = 1
LINEITEM_COLS = ("qty", "price", "disc", "tax", "shipdate", "flag1", "flag2")


def lineitem_to_device(cols: dict, device="cuda") -> dict:
    return {k: torch.from_numpy(np.ascontiguousarray(cols[k])).to(device) for k in LINEITEM_COLS}


def filter_groupby_scratch_bytes(n: int, group_bound: int) -> int:
    return int(lib().velo_filter_groupby_scratch_bytes(n, group_bound))


def filter_groupby(dcols: dict, n: int, pred: dict, group_bound: int = 8, reveal_count: bool = False,
                   scratch=None, out=None, counts=None, stream=None):
    """Oblivious filter + group-by (velo_filter_groupby).  Returns the device
    tensors (out[group_bound, 6] int64, counts[2] int64)."""
    from ._lib import VeloLineitem, VeloLineitemPred

    dev = dcols["qty"].device
    cols = VeloLineitem(*[dcols[k].data_ptr() for k in LINEITEM_COLS])
    p = VeloLineitemPred(*[int(pred[k]) for k in ("ship_lo", "ship_hi", "disc_lo", "disc_hi", "qty_lo", "qty_hi")])
    if scratch is None:
        scratch = torch.empty(filter_groupby_scratch_bytes(n, group_bound), dtype=torch.uint8, device=dev)
    if out is None:
        out = torch.empty((group_bound, 6), dtype=torch.int64, device=dev)
    if counts is None:
        counts = torch.empty(2, dtype=torch.int64, device=dev)
    import ctypes as C

    check(lib().velo_filter_groupby(C.byref(cols), n, C.byref(p), group_bound, REVEAL_COUNT if reveal_count else 0,
                                    out.data_ptr(), counts.data_ptr(), scratch.data_ptr(), scratch.numel(),
                                    _stream(stream)), "velo_filter_groupby")
    return out, counts


def join_to_device(dim: dict, fact: dict, device="cuda") -> dict:
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(device)  # noqa: E731
    return dict(dim_key=t(dim["key"]), dim_date=t(dim["date"]), fact_fk=t(fact["fk"]), fact_price=t(fact["price"]))


def join_groupby_topk_scratch_bytes(n_dim: int, n_fact: int) -> int:
    return int(lib().velo_join_groupby_topk_scratch_bytes(n_dim, n_fact))


def join_groupby_topk(dt: dict, pred: dict, k: int = 10, scratch=None, out=None, counts=None, stream=None):
    """Oblivious PK-FK join + group-by + top-k (velo_join_groupby_topk).
    Returns device tensors out[k, 3] (fk, sum, count) and counts[2]."""
    import ctypes as C

    from ._lib import VeloJoinPred, VeloJoinTables

    nd, nf = dt["dim_key"].numel(), dt["fact_fk"].numel()
    dev = dt["dim_key"].device
    tabs = VeloJoinTables(dt["dim_key"].data_ptr(), dt["dim_date"].data_ptr(), nd, dt["fact_fk"].data_ptr(),
                          dt["fact_price"].data_ptr(), nf)
    p = VeloJoinPred(int(pred["date_hi"]), 0, int(pred["price_hi"]))
    if scratch is None:
        scratch = torch.empty(join_groupby_topk_scratch_bytes(nd, nf), dtype=torch.uint8, device=dev)
    if out is None:
        out = torch.empty((k, 3), dtype=torch.int64, device=dev)
    if counts is None:
        counts = torch.empty(2, dtype=torch.int64, device=dev)
    check(lib().velo_join_groupby_topk(C.byref(tabs), C.byref(p), k, out.data_ptr(), counts.data_ptr(),
                                       scratch.data_ptr(), scratch.numel(), _stream(stream)),
          "velo_join_groupby_topk")
    return out, counts


SORT_STRICT = 1


def osort_records(words, n: int, key_mask: int, strict: bool = False, tune=None, stream=None) -> None:
    """In-place oblivious sort of 1..3-word records (velo_osort_records);
    `words` are int64 device tensors of equal capacity (SoA)."""
    ptrs = np.asarray([w.data_ptr() for w in words], dtype=np.uint64)
    cap = min(w.numel() for w in words)
    check(lib().velo_osort_records(ptrs.ctypes.data, len(words), key_mask & 0xFFFFFFFFFFFFFFFF, n, cap,
                                   SORT_STRICT if strict else 0, tune_ref(tune), _stream(stream)),
          "velo_osort_records")


ITEM_SORT_KP, ITEM_COMPACT_KPM = 1, 2


class Batch:
    """A planned batch of sorts/compactions run by one persistent launch
    (velo_batch_*).  items: list of dicts with kind ('sort'|'compact'),
    keys/pay/marks device tensors, n, and for compactions a count tensor."""

    def __init__(self, items, tune=None):
        import ctypes as C

        from ._lib import VeloBatchItem

        arr = (VeloBatchItem * max(1, len(items)))()
        for i, it in enumerate(items):
            kind = ITEM_SORT_KP if it["kind"] == "sort" else ITEM_COMPACT_KPM
            cap = min(it["keys"].numel(), it["pay"].numel())
            marks = it.get("marks")
            cnt = it.get("count")
            if marks is not None:
                cap = min(cap, marks.numel())
            arr[i] = VeloBatchItem(kind, 0, it["keys"].data_ptr(), it["pay"].data_ptr(),
                                   marks.data_ptr() if marks is not None else None, it["n"], cap,
                                   cnt.data_ptr() if cnt is not None else None)
        self._arr = arr
        self._n = len(items)
        self.ptr = C.c_void_p()
        check(lib().velo_batch_create(arr, len(items), tune_ref(tune), C.byref(self.ptr)), "velo_batch_create")

    def launch(self, stream=None):
        check(lib().velo_batch_launch(self.ptr, _stream(stream)), "velo_batch_launch")

    def status(self, stream=None):
        check(lib().velo_batch_status(self.ptr, _stream(stream)), "velo_batch_status")

    def close(self):
        if self.ptr:
            lib().velo_batch_destroy(self.ptr)
            self.ptr = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def batch_autotune(items, reps=2, stream=None):
    """Runs the autotuner over the 9 tile configurations; returns
    ((tile_log2, threads), {config: ms})."""
    import ctypes as C

    from ._lib import VeloTune

    b = Batch(items)  # only to marshal the item array
    best = VeloTune(0, 0)
    ms = (C.c_float * 9)()
    check(lib().velo_batch_autotune(b._arr, b._n, reps, C.byref(best), ms, _stream(stream)), "velo_batch_autotune")
    b.close()
    cands = [(11, 256), (11, 512), (11, 1024), (12, 256), (12, 512), (12, 1024), (13, 256), (13, 512), (13, 1024)]
    return (best.tile_log2, best.threads), {c: float(m) for c, m in zip(cands, ms)}


def _ptr(t):
    return t.data_ptr() if t is not None else None


def _scratch(nbytes, device):
    return torch.empty(max(int(nbytes), 1), dtype=torch.uint8, device=device)


def permute(out, inp, idx, n, type_id, stream=None):
    check(lib().velo_permute(out.data_ptr(), inp.data_ptr(), idx.data_ptr(), n, type_id, _stream(stream)),
          "velo_permute")


def scatter(mask, n, out_idx, stream=None):
    cnt = torch.zeros(1, dtype=torch.int64, device=mask.device)
    sc = _scratch(lib().velo_scatter_scratch_bytes(n), mask.device)
    check(lib().velo_scatter(mask.data_ptr(), n, out_idx.data_ptr(), cnt.data_ptr(), sc.data_ptr(), sc.numel(),
                             _stream(stream)), "velo_scatter")
    return cnt


def gather(out, inp, idx, mask, n, type_id, stream=None):
    check(lib().velo_gather(out.data_ptr(), inp.data_ptr(), idx.data_ptr(), _ptr(mask), n, type_id, _stream(stream)),
          "velo_gather")


def compare_eq(left, right, out, n, type_id, stream=None):
    check(lib().velo_compare_eq(left.data_ptr(), right.data_ptr(), out.data_ptr(), n, type_id, _stream(stream)),
          "velo_compare_eq")


def compose_position_map(old, sigma, new, n, stream=None):
    check(lib().velo_compose_position_map(old.data_ptr(), sigma.data_ptr(), new.data_ptr(), n, _stream(stream)),
          "velo_compose_position_map")


def enrich_positions(rids, pmap, out, n, stream=None):
    check(lib().velo_enrich_positions(rids.data_ptr(), pmap.data_ptr(), out.data_ptr(), n, _stream(stream)),
          "velo_enrich_positions")


def oshuffle_position_map(pmap, n, key, counter, stream=None):
    sc = _scratch(lib().velo_oshuffle_scratch_bytes(n), pmap.device)
    check(lib().velo_oshuffle_position_map(pmap.data_ptr(), n, key & (2**64 - 1), counter & (2**64 - 1),
                                           sc.data_ptr(), sc.numel(), _stream(stream)), "velo_oshuffle_position_map")


def ogather_u64(table, table_n, rids, n_req, out, stream=None):
    sc = _scratch(lib().velo_ogather_scratch_bytes(table_n, n_req), table.device)
    check(lib().velo_ogather_u64(table.data_ptr(), table_n, rids.data_ptr(), n_req, out.data_ptr(), sc.data_ptr(),
                                 sc.numel(), _stream(stream)), "velo_ogather_u64")


def ojoin_pkfk(build_keys, build_mask, probe_keys, probe_mask, key_type, stream=None):
    """Returns (build rowids, probe rowids, counts[2]) device tensors; rows
    past counts[0] are -1."""
    bn, pn = build_keys.numel(), probe_keys.numel()
    dev = build_keys.device
    ob = torch.empty(max(pn, 1), dtype=torch.int64, device=dev)
    op = torch.empty(max(pn, 1), dtype=torch.int64, device=dev)
    cnt = torch.zeros(2, dtype=torch.int64, device=dev)
    sc = _scratch(lib().velo_ojoin_scratch_bytes(bn, pn), dev)
    check(lib().velo_ojoin_pkfk(build_keys.data_ptr(), _ptr(build_mask), bn, probe_keys.data_ptr(), _ptr(probe_mask),
                                pn, key_type, ob.data_ptr(), op.data_ptr(), cnt.data_ptr(), sc.data_ptr(), sc.numel(),
                                _stream(stream)), "velo_ojoin_pkfk")
    return ob, op, cnt


def ojoin_mn(build_keys, build_mask, probe_keys, probe_mask, key_type, max_pairs, stream=None):
    """Oblivious many-to-many equi-join (velo_ojoin_mn).  Returns (build
    rowids, probe rowids, counts[2] = (pairs, overflow)) device tensors of
    max_pairs rows; rows past the pair count are -1."""
    bn, pn = build_keys.numel(), probe_keys.numel()
    dev = build_keys.device
    ob = torch.empty(max_pairs, dtype=torch.int64, device=dev)
    op = torch.empty(max_pairs, dtype=torch.int64, device=dev)
    cnt = torch.zeros(2, dtype=torch.int64, device=dev)
    sc = _scratch(lib().velo_ojoin_mn_scratch_bytes(bn, pn, max_pairs), dev)
    check(lib().velo_ojoin_mn(build_keys.data_ptr(), _ptr(build_mask), bn, probe_keys.data_ptr(), _ptr(probe_mask),
                              pn, key_type, max_pairs, ob.data_ptr(), op.data_ptr(), cnt.data_ptr(), sc.data_ptr(),
                              sc.numel(), _stream(stream)), "velo_ojoin_mn")
    return ob, op, cnt


def ohash_join(build_keys, build_mask, probe_keys, probe_mask, key_type, hash_seed=0x5EED, stream=None):
    """Oblivious bin-padded hash join (velo_ohash_join).  Returns (build
    rowids, probe rowids, counts[3] = (pairs, repeated build keys, overflowed
    rows)) device tensors of probe_n rows."""
    bn, pn = build_keys.numel(), probe_keys.numel()
    dev = build_keys.device
    ob = torch.empty(max(pn, 1), dtype=torch.int64, device=dev)
    op = torch.empty(max(pn, 1), dtype=torch.int64, device=dev)
    cnt = torch.zeros(3, dtype=torch.int64, device=dev)
    sc = _scratch(lib().velo_ohash_join_scratch_bytes(bn, pn), dev)
    check(lib().velo_ohash_join(build_keys.data_ptr(), _ptr(build_mask), bn, probe_keys.data_ptr(),
                                _ptr(probe_mask), pn, key_type, hash_seed, ob.data_ptr(), op.data_ptr(),
                                cnt.data_ptr(), sc.data_ptr(), sc.numel(), _stream(stream)), "velo_ohash_join")
    return ob, op, cnt


def ogroupby(keys: torch.Tensor, key_type: int, n: int, sums=(), with_count: bool = True, mask=None,
             group_bound: int | None = None, stream=None):
    """Oblivious GROUP BY key with SUM/COUNT (velo_ogroupby).  keys: int32
    (key_type 4) or int64 (5) device tensor; sums: up to two int64 device
    tensors (one when with_count).  Returns (out_keys, [out_sums], out_counts
    or None, counts[2] = (groups, rows left out for their key)) as device
    tensors of group_bound rows (default n)."""
    import ctypes as C

    dev = keys.device
    bound = n if group_bound is None else group_bound
    out_keys = torch.empty(max(bound, 1), dtype=torch.int64, device=dev)
    out_sums = [torch.empty(max(bound, 1), dtype=torch.int64, device=dev) for _ in sums]
    out_counts = torch.empty(max(bound, 1), dtype=torch.int64, device=dev) if with_count else None
    counts = torch.empty(2, dtype=torch.int64, device=dev)
    nb = int(lib().velo_ogroupby_scratch_bytes(n))
    scratch = torch.empty(max(nb, 1), dtype=torch.uint8, device=dev)
    sp = (C.c_void_p * 2)(*[s.data_ptr() for s in sums], *([None] * (2 - len(sums))))
    op = (C.c_void_p * 2)(*[s.data_ptr() for s in out_sums], *([None] * (2 - len(sums))))
    check(lib().velo_ogroupby(keys.data_ptr(), key_type, sp, len(sums), 1 if with_count else 0,
                              mask.data_ptr() if mask is not None else None, n, bound, out_keys.data_ptr(), op,
                              out_counts.data_ptr() if out_counts is not None else None, counts.data_ptr(),
                              scratch.data_ptr(), scratch.numel(), _stream(stream)), "velo_ogroupby")
    return out_keys, out_sums, out_counts, counts


# ---- command queue (velo_init / velo_submit / velo_wait) ----------------------------

QUEUE_PERSISTENT = 1
CMD_UNORDERED = 0x100


def make_cmd(opcode: str, *fields, flags: int = 0):
    """A velo_cmd for `opcode` (a key of _lib.OP) with the union member's
    fields in declaration order (pointers as ints or tensors)."""
    from ._lib import OP, VeloCmd

    member = {"OSORT_KP": "osort_kp", "OCOMPACT_KPM": "ocompact_kpm", "PERMUTE": "permute", "GATHER": "gather",
              "COMPARE_EQ": "compare_eq", "COMPOSE_POSITION_MAP": "compose", "ENRICH_POSITIONS": "enrich",
              "SCATTER": "scatter", "OSHUFFLE": "oshuffle", "OJOIN_PKFK": "ojoin", "OGATHER": "ogather",
              "FILTER_GROUPBY": "filter_groupby", "JOIN_GROUPBY_TOPK": "join_topk", "OJOIN_MN": "ojoin_mn",
              "OHASH_JOIN": "ohash"}.get(opcode)
    m = VeloCmd()
    m.opcode = OP[opcode]
    m.flags = flags
    if member is not None:
        a = getattr(m.args, member)
        for i, v in enumerate(fields):
            if torch.is_tensor(v):
                v = v.data_ptr()
            setattr(a, f"f{i}", 0 if v is None else v)
    return m


class Queue:
    """A command queue context (velo_init): the stream queue, or with
    persistent=True the persistent device consumer.  The queue is not ordered
    after torch's streams: tensors a command reads or writes must be ready
    (e.g. torch.cuda.synchronize()) before it is submitted."""

    def __init__(self, device: int = 0, persistent: bool = False, idle_us: int = 0, capacity: int = 0):
        import ctypes as C

        from ._lib import VeloConfig

        self._c = C.c_void_p()
        cfg = VeloConfig(device, capacity, QUEUE_PERSISTENT if persistent else 0, idle_us)
        check(lib().velo_init(C.byref(cfg), C.byref(self._c)), "velo_init")

    def submit(self, cmd) -> int:
        import ctypes as C

        t = C.c_uint64()
        check(lib().velo_submit(self._c, C.byref(cmd), C.byref(t)), "velo_submit")
        return t.value

    def submit_raw(self, cmd) -> int:
        """velo_submit's status, for tests of rejected commands."""
        import ctypes as C

        t = C.c_uint64()
        return int(lib().velo_submit(self._c, C.byref(cmd), C.byref(t)))

    def submit_batch(self, cmds) -> list:
        import ctypes as C

        from ._lib import VeloCmd

        arr = (VeloCmd * len(cmds))(*cmds)
        tix = (C.c_uint64 * len(cmds))()
        check(lib().velo_batch_submit(self._c, arr, len(cmds), tix), "velo_batch_submit")
        return list(tix)

    def wait(self, ticket: int, timeout_s: float = 30.0) -> None:
        check(lib().velo_wait(self._c, ticket, int(timeout_s * 1e9)), "velo_wait")

    def wait_raw(self, ticket: int, timeout_ns: int) -> int:
        return int(lib().velo_wait(self._c, ticket, timeout_ns))

    def launches(self) -> int:
        return int(lib().velo_ctx_launches(self._c))

    def close(self, timeout_ms: int = 30_000) -> None:
        if self._c:
            c, self._c = self._c, None
            check(lib().velo_shutdown(c, timeout_ms), "velo_shutdown")

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
