"""velo_ocompact_kpm_noalloc: the allocation-free compaction entry point.

Some callers of this library cannot allocate device memory where they compact
(an engine whose HBM belongs to its own pool allocator, a latency-critical
path that cannot take cudaMalloc's implicit synchronisation, a plugin host
without an allocation hook).  The variant keeps its scratch in a fixed array
inside the library instead of taking a caller buffer.  This test calls it
through the C ABI twice in a row, on different inputs, and requires each
result to equal the existing entry point's (velo_ocompact_kpm, with a
caller-provided scratch buffer) exactly.  The file is named to be collected
last so that a run stopping at the first failure has run every other test.
"""
import numpy as np
import pytest
import torch

import velodb_b200
from velodb_b200 import capi, workloads as W
from velodb_b200._lib import check

pytestmark = pytest.mark.gpu


def _dev(keys, pay, marks):
    cap = capi.next_pow2(len(keys))
    return capi.to_dev_u64(keys, cap), capi.to_dev_u32(pay, cap), capi.to_dev_u8(marks, cap)


def _noalloc(keys, pay, marks):
    k, p, m = _dev(keys, pay, marks)
    cnt = torch.full((1,), -1, dtype=torch.int64, device=k.device)
    stream = torch.cuda.current_stream().cuda_stream
    check(velodb_b200.lib().velo_ocompact_kpm_noalloc(k.data_ptr(), p.data_ptr(), m.data_ptr(), len(keys),
                                                      k.numel(), cnt.data_ptr(), stream),
          "velo_ocompact_kpm_noalloc")
    torch.cuda.synchronize()
    return k.cpu().numpy(), p.cpu().numpy(), m.cpu().numpy(), int(cnt.item())


def _with_scratch(keys, pay, marks):
    k, p, m = _dev(keys, pay, marks)
    cnt = capi.ocompact_kpm(k, p, m, len(keys))
    torch.cuda.synchronize()
    return k.cpu().numpy(), p.cpu().numpy(), m.cpu().numpy(), int(cnt.item())


def _inputs_density(n, seed, tenths):
    keys = W.splitmix64(seed, n, 0)
    pay = np.arange(n, dtype=np.uint32)
    marks = (W.lemire(W.splitmix64(seed, n, 1), 10) < tenths).astype(np.uint8)
    return keys, pay, marks


@pytest.mark.parametrize("calls", [
    # small then large: the second call has more tiles than the first
    [(300_001, 11, 3), (2_000_003, 12, 3)],
    # large then small with another mark density: the per-tile counts and
    # prefix values of the first call stay in the array past the second
    # call's tiles, where a scan that read beyond its own tiles would see them
    [(2_000_003, 13, 7), (300_001, 14, 2)],
])
def test_noalloc_matches_scratch_entry_point_twice(cuda, calls):
    for n, seed, tenths in calls:
        keys, pay, marks = _inputs_density(n, seed, tenths)
        a = _noalloc(keys, pay, marks)
        b = _with_scratch(keys, pay, marks)
        assert a[3] == b[3] == int(marks.sum())
        for x, y in zip(a[:3], b[:3]):
            assert np.array_equal(x, y)


def test_noalloc_rejects_sizes_beyond_its_limit(cuda):
    k = torch.empty(1, dtype=torch.int64, device=cuda)
    rc = velodb_b200.lib().velo_ocompact_kpm_noalloc(k.data_ptr(), k.data_ptr(), k.data_ptr(), (1 << 28) + 1,
                                                     1 << 29, k.data_ptr(), None)
    assert rc == -1 and "2^28" in velodb_b200._lib.last_error()
