"""GPU tests of the batched form: one persistent launch for many sorts and
compactions must give, command by command, exactly the plain path's result;
it must capture into a CUDA graph; its bounded waits must end a launch whose
dependency is never met with VELO_ETIMEDOUT instead of hanging."""
import numpy as np
import pytest
import torch

import velodb_b200
from velodb_b200 import capi, workloads as W
from velodb_b200._lib import check

pytestmark = pytest.mark.gpu


def make_items(sizes, seed, device):
    items = []
    for i, n in enumerate(sizes):
        cap = capi.next_pow2(max(n, 1))
        keys = W.splitmix64(seed, n, 2 * i)
        it = dict(kind="sort" if i % 2 == 0 else "compact", n=n, keys=capi.to_dev_u64(keys, cap),
                  pay=capi.to_dev_u32(np.arange(n, dtype=np.uint32), cap))
        if it["kind"] == "compact":
            marks = (W.lemire(W.splitmix64(seed, n, 2 * i + 1), 10) < 3).astype(np.uint8)
            it["marks"] = capi.to_dev_u8(marks, cap)
            it["count"] = torch.full((1,), -1, dtype=torch.int64, device=device)
        items.append(it)
    return items


def clone_items(items):
    out = []
    for it in items:
        c = dict(it)
        for k in ("keys", "pay", "marks", "count"):
            if k in c:
                c[k] = it[k].clone()
        out.append(c)
    return out


def run_plain(items, tune):
    for it in items:
        if it["kind"] == "sort":
            capi.osort_kp(it["keys"], it["pay"], it["n"], tune=tune)
        else:
            it["count"].copy_(capi.ocompact_kpm(it["keys"], it["pay"], it["marks"], it["n"], tune=tune))
    torch.cuda.synchronize()


def assert_same(a_items, b_items):
    for a, b in zip(a_items, b_items):
        n = capi.next_pow2(max(a["n"], 1)) if a["n"] else 0
        for k in ("keys", "pay", "marks"):
            if k in a and n:
                assert torch.equal(a[k][:n], b[k][:n]), (a["kind"], a["n"], k)
        if "count" in a:
            assert int(a["count"].item()) == int(b["count"].item())


SIZES = [0, 1, 2, 3, 1000, 1024, 5000, 8191, 8193, 40_000, 65_536, 100_000, 300_001, 1 << 20, 7, 12_345]


@pytest.mark.parametrize("tune", [(13, 512), (11, 256), (12, 1024), (13, 1024)])
def test_batch_matches_plain_path(cuda, tune):
    items = make_items(SIZES, 31, cuda)
    ref = clone_items(items)
    run_plain(ref, tune)
    b = capi.Batch(items, tune=tune)
    b.launch()
    b.status()
    assert_same(items, ref)
    b.close()


def test_batch_matches_oracle(cuda, orc):
    items = make_items([777, 4096, 50_000, 3], 5, cuda)
    host = [(capi.host_u64(it["keys"], it["n"]).copy(), capi.host_u32(it["pay"], it["n"]).copy()) for it in items]
    b = capi.Batch(items)
    b.launch()
    b.status()
    for it, (k, p) in zip(items, host):
        if it["kind"] == "sort":
            ok, op = orc.bitonic_kp(k, p)
            n = len(ok)
            assert np.array_equal(capi.host_u64(it["keys"], n), ok)
            assert np.array_equal(capi.host_u32(it["pay"], n), op)
        else:
            m = it["marks"].cpu().numpy()  # compacted marks: first count set
            cnt = int(it["count"].item())
            assert m[:cnt].all() and not m[cnt:].any()


def test_batch_graph_capture_and_replay(cuda):
    items = make_items([10_000, 70_000, 300_000, 5_000], 77, cuda)
    ref = clone_items(items)
    run_plain(ref, None)
    b = capi.Batch(items)
    b.launch()  # first launch outside the graph (sets up the kernel)
    b.status()
    # restore the inputs, then capture and replay
    fresh = make_items([10_000, 70_000, 300_000, 5_000], 77, cuda)
    for it, f in zip(items, fresh):
        for k in ("keys", "pay", "marks"):
            if k in it:
                it[k].copy_(f[k])
    s = torch.cuda.Stream()
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=s):
        b.launch(stream=s)
    g.replay()
    torch.cuda.synchronize()
    assert_same(items, ref)
    # a second replay re-sorts sorted rows (same output) and re-compacts
    # compacted rows (same marked prefix and count; the unmarked tail is
    # re-routed, since rows past n are re-padded)
    g.replay()
    torch.cuda.synchronize()
    for a, r in zip(items, ref):
        n = capi.next_pow2(a["n"])
        if a["kind"] == "sort":
            assert torch.equal(a["keys"][:n], r["keys"][:n]) and torch.equal(a["pay"][:n], r["pay"][:n])
        else:
            c = int(r["count"].item())
            assert int(a["count"].item()) == c
            assert torch.equal(a["keys"][:c], r["keys"][:c]) and torch.equal(a["pay"][:c], r["pay"][:c])
    del g
    b.close()


def test_batch_bounded_wait_reports_timeout(cuda):
    items = make_items([5000, 20_000, 3000], 3, cuda)
    b = capi.Batch(items)
    L = velodb_b200.lib()
    check(L.velo_batch_set_timeout(b.ptr, 2_000_000), "velo_batch_set_timeout")  # 2 ms
    check(L.velo_batch_inject_unmet_wait(b.ptr, 1), "velo_batch_inject_unmet_wait")
    b.launch()
    with pytest.raises(velodb_b200.VeloError) as e:
        b.status()
    assert e.value.status == -4  # VELO_ETIMEDOUT
    b.close()
    # the device stays usable
    items = make_items([5000], 4, cuda)
    b = capi.Batch(items)
    b.launch()
    b.status()
    b.close()


def test_batch_autotune(cuda):
    items = make_items([2000, 30_000, 200_000, 1 << 20], 9, cuda)
    best, ms = capi.batch_autotune(items, reps=1)
    assert best in ms and ms[best] == min(ms.values())
