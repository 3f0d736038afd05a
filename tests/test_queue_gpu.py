"""GPU tests of the command queue (velo_init / velo_submit / velo_batch_submit
/ velo_wait / velo_shutdown): commands give the same results as the direct
entry points, tickets complete in order, waits are bounded."""
import ctypes as C

import numpy as np
import pytest
import torch

import velodb_b200
from velodb_b200 import capi, workloads as W
from velodb_b200._lib import OP, VeloCmd, VeloConfig, check

pytestmark = pytest.mark.gpu


@pytest.fixture
def ctx(cuda):
    L = velodb_b200.lib()
    c = C.c_void_p()
    check(L.velo_init(C.byref(VeloConfig(0, 16)), C.byref(c)), "velo_init")
    yield c
    check(L.velo_shutdown(c, 10_000), "velo_shutdown")


def sort_cmd(k, p, n):
    m = VeloCmd()
    m.opcode = OP["OSORT_KP"]
    a = m.args.osort_kp
    a.f0, a.f1, a.f2, a.f3 = k.data_ptr(), p.data_ptr(), n, min(k.numel(), p.numel())
    return m


def compact_cmd(k, p, mk, n, cnt, scratch):
    m = VeloCmd()
    m.opcode = OP["OCOMPACT_KPM"]
    a = m.args.ocompact_kpm
    a.f0, a.f1, a.f2, a.f3, a.f4 = k.data_ptr(), p.data_ptr(), mk.data_ptr(), n, min(k.numel(), p.numel(), mk.numel())
    a.f5, a.f6, a.f7 = cnt.data_ptr(), scratch.data_ptr(), scratch.numel()
    return m


def test_cmd_layout_matches_library():
    assert C.sizeof(VeloCmd) == velodb_b200.lib().velo_cmd_size()


def test_submit_and_wait_matches_direct_calls(ctx, orc):
    L = velodb_b200.lib()
    tickets = []
    cases = []
    for i, n in enumerate([1000, 70_000, 300_001]):
        keys, pay = W.sort_kp(n, seed=500 + i)
        cap = capi.next_pow2(n)
        k, p = capi.to_dev_u64(keys, cap), capi.to_dev_u32(pay, cap)
        t = C.c_uint64()
        check(L.velo_submit(ctx, C.byref(sort_cmd(k, p, n)), C.byref(t)), "velo_submit")
        tickets.append(t.value)
        cases.append((keys, pay, k, p))
    assert tickets == sorted(tickets)
    for t in reversed(tickets):
        check(L.velo_wait(ctx, t, 10_000_000_000), "velo_wait")
    for keys, pay, k, p in cases:
        ok, op = orc.bitonic_kp(keys, pay)
        assert np.array_equal(capi.host_u64(k, len(ok)), ok) and np.array_equal(capi.host_u32(p, len(op)), op)


def test_batch_submit_runs_one_persistent_launch(ctx):
    L = velodb_b200.lib()
    cmds, refs, keep = [], [], []
    for i, n in enumerate([3000, 20_000, 150_000, 9000]):
        cap = capi.next_pow2(n)
        keys = W.splitmix64(900 + i, n, 0)
        k, p = capi.to_dev_u64(keys, cap), capi.to_dev_u32(np.arange(n, dtype=np.uint32), cap)
        if i % 2 == 0:
            cmds.append(sort_cmd(k, p, n))
            refs.append(("sort", np.sort(keys), k))
        else:
            marks = (W.lemire(W.splitmix64(900 + i, n, 1), 10) < 3).astype(np.uint8)
            mk = capi.to_dev_u8(marks, cap)
            cnt = torch.zeros(1, dtype=torch.int64, device="cuda")
            sc = torch.empty(capi.compact_scratch_bytes(cap), dtype=torch.uint8, device="cuda")
            cmds.append(compact_cmd(k, p, mk, n, cnt, sc))
            refs.append(("compact", keys[marks.astype(bool)], k, cnt))
            keep += [mk, sc]
        keep += [k, p]
    arr = (VeloCmd * len(cmds))(*cmds)
    tix = (C.c_uint64 * len(cmds))()
    check(L.velo_batch_submit(ctx, arr, len(cmds), tix), "velo_batch_submit")
    check(L.velo_wait(ctx, tix[0], 10_000_000_000), "velo_wait")
    for r in refs:
        if r[0] == "sort":
            assert np.array_equal(capi.host_u64(r[2], len(r[1])), r[1])
        else:
            c = int(r[3].item())
            assert c == len(r[1]) and np.array_equal(capi.host_u64(r[2], c), r[1])


def test_wait_is_bounded(ctx):
    L = velodb_b200.lib()
    n = 1 << 24
    keys, pay = W.sort_kp(n, seed=1)
    k, p = capi.to_dev_u64(keys), capi.to_dev_u32(pay)
    t = C.c_uint64()
    check(L.velo_submit(ctx, C.byref(sort_cmd(k, p, n)), C.byref(t)), "velo_submit")
    rc = L.velo_wait(ctx, t.value, 1000)  # 1 us: the sort cannot be done yet
    assert rc == -4  # VELO_ETIMEDOUT
    check(L.velo_wait(ctx, t.value, 30_000_000_000), "velo_wait")
    buf = C.create_string_buffer(256)
    check(L.velo_last_error(ctx, buf, 256), "velo_last_error")
    assert b"time limit" in buf.value


def test_unknown_opcode_and_ticket(ctx):
    L = velodb_b200.lib()
    m = VeloCmd()
    m.opcode = 0x7777
    t = C.c_uint64()
    assert L.velo_submit(ctx, C.byref(m), C.byref(t)) == -1
    assert L.velo_wait(ctx, 10**9, 1000) == -1
