"""CPU tests of the C ABI: the library loads without a GPU, exports every
function declared in include/*.h, and validates arguments before touching the
device."""
import ctypes as C
import glob
import os
import re

import numpy as np

import velodb_b200
from velodb_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"\b(velo_[a-z0-9_]+)\s*\(", text):
            names.add(m.group(1))
    return names


def test_library_exports_every_declared_function():
    L = velodb_b200.lib()
    names = declared_functions()
    assert len(names) >= 5
    missing = [n for n in sorted(names) if not hasattr(L, n)]
    assert not missing, f"declared but not exported: {missing}"
    # every declared function has a ctypes prototype in the Python loader
    assert not (names - set(_lib.PROTOS)), names - set(_lib.PROTOS)


def test_next_pow2():
    L = velodb_b200.lib()
    for x, e in [(0, 1), (1, 1), (2, 2), (3, 4), (1000, 1024), (1 << 20, 1 << 20), ((1 << 20) + 1, 1 << 21)]:
        assert L.velo_next_pow2(x) == e


def test_argument_validation_without_gpu():
    L = velodb_b200.lib()
    k = np.zeros(8, np.uint64)
    p = np.zeros(8, np.uint32)
    # capacity below next_pow2(n) is rejected before any launch
    rc = L.velo_osort_kp(k.ctypes.data, p.ctypes.data, 5, 4, None, None)
    assert rc == -1 and "capacity" in _lib.last_error()
    rc = L.velo_osort_kp(None, None, 5, 8, None, None)
    assert rc == -1
    t = _lib.VeloTune(12, 300)
    rc = L.velo_osort_kp(k.ctypes.data, p.ctypes.data, 5, 8, C.byref(t), None)
    assert rc == -1 and "power of two" in _lib.last_error()
    # zero rows is a no-op
    assert L.velo_osort_kp(k.ctypes.data, p.ctypes.data, 0, 0, None, None) == 0
    # compaction without enough scratch
    m = np.zeros(8, np.uint8)
    cnt = np.zeros(1, np.uint64)
    rc = L.velo_ocompact_kpm(k.ctypes.data, p.ctypes.data, m.ctypes.data, 5, 8, cnt.ctypes.data, None, 0, None, None)
    assert rc == -2


def test_compact_scratch_size():
    L = velodb_b200.lib()
    small = L.velo_compact_scratch_bytes(1000, None)
    big = L.velo_compact_scratch_bytes(1 << 23, None)
    assert 0 < small <= big
    # one u32 count and one u32 prefix per 4096-row tile (the default tiles
    # above 2^18 rows and the persistent queue's), 256-byte aligned
    assert big == 2 * ((1 << 11) * 4) + 256
    # up to 2^18 rows the default tiles hold 2048 rows: 128 of them
    assert L.velo_compact_scratch_bytes(1 << 18, None) == 512 + 768  # 128 counts, 129 prefix words
    # with an explicit tune: that tune's tiles only (8192 rows here)
    t = _lib.VeloTune(13, 512)
    assert L.velo_compact_scratch_bytes(1 << 23, C.byref(t)) == 2 * ((1 << 10) * 4) + 256


def test_queue_init_without_device_fails_cleanly():
    import torch

    if torch.cuda.is_available():
        return  # covered by tests/test_queue_gpu.py on a GPU
    L = velodb_b200.lib()
    c = C.c_void_p()
    rc = L.velo_init(C.byref(_lib.VeloConfig(0, 8)), C.byref(c))
    assert rc == -3 and not c.value  # VELO_ECUDA, no context
    assert L.velo_shutdown(None, 0) == 0
    buf = C.create_string_buffer(64)
    assert L.velo_last_error(None, buf, 64) == 0
