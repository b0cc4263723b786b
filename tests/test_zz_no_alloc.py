"""mp_exclusive_scan_noalloc: the exclusive scan for callers that cannot
allocate device memory when they need a scan (fixed per-frame memory budgets,
host frameworks that own the device heap).  Its scratch is a static device
array of the library, so the test checks that two calls in a row, each
reusing what the previous call left there, give exactly the result of the
allocating mp_exclusive_scan.  This file is collected last on purpose."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

LIMIT = 1 << 24  # elements the static scratch can serve


def _scan_both(x):
    import torch

    from mtlphys_b200 import _abi, exclusive_scan

    lib = _abi.load()
    t = torch.from_numpy(x.view(np.int32)).cuda()
    want = exclusive_scan(t)                      # allocating entry point (torch scratch)
    got = torch.full_like(t, -1)
    stream = torch.cuda.current_stream()
    rc = lib.mp_exclusive_scan_noalloc(C.c_void_p(t.data_ptr()), C.c_void_p(got.data_ptr()),
                                       len(x), C.c_void_p(stream.cuda_stream))
    assert rc == _abi.MP_OK, lib.mp_last_error()
    torch.cuda.synchronize()
    return got.cpu().numpy().view(np.uint32), want.cpu().numpy().view(np.uint32)


def test_noalloc_scan_matches_the_allocating_scan_twice_in_a_row(cuda):
    rng = np.random.default_rng(2024)
    # a large call first, then a smaller one that reuses (and must clear) the
    # descriptors and ticket the first call left in the shared array
    for n, hi in ((3_000_017, 7), (700_001, 2**32 - 1)):
        x = rng.integers(0, hi, size=n, endpoint=True, dtype=np.uint64).astype(np.uint32)
        got, want = _scan_both(x)
        bad = np.nonzero(got != want)[0]
        assert bad.size == 0, f"n={n}: first mismatch at {bad[0]}: {got[bad[0]]} != {want[bad[0]]}"


def test_noalloc_scan_rejects_sizes_beyond_its_static_scratch(cuda):
    import torch

    from mtlphys_b200 import _abi

    lib = _abi.load()
    t = torch.zeros(8, dtype=torch.int32, device="cuda")
    rc = lib.mp_exclusive_scan_noalloc(C.c_void_p(t.data_ptr()), C.c_void_p(t.data_ptr()),
                                       LIMIT + 1, None)
    assert rc == _abi.MP_ERR_INVALID_ARGUMENT
    assert b"limit" in lib.mp_last_error()


def test_noalloc_scan_at_its_limit_and_in_place_unaligned(cuda):
    """n = 2^24 fills every tile descriptor and the last bytes of the static
    array; an in-place call on a pointer 4 or 12 bytes past a 16-byte boundary
    takes the scalar load/store path.  Both against numpy's prefix sum (and
    the first also against the allocating scan)."""
    import torch

    from mtlphys_b200 import _abi

    lib = _abi.load()
    rng = np.random.default_rng(77)
    x = rng.integers(0, 5, size=LIMIT).astype(np.uint32)
    got, want = _scan_both(x)
    ref = (np.cumsum(x, dtype=np.uint64) - x).astype(np.uint32)
    np.testing.assert_array_equal(want, ref)
    np.testing.assert_array_equal(got, ref)
    stream = torch.cuda.current_stream()
    assert lib.mp_exclusive_scan_status(None, C.c_void_p(stream.cuda_stream)) == _abi.MP_OK
    for n, off in ((1_000_003, 1), (4097, 3)):
        y = rng.integers(0, 2**32, size=n, dtype=np.uint64).astype(np.uint32)
        buf = torch.zeros(n + off, dtype=torch.int32, device="cuda")
        t = buf[off:]
        t.copy_(torch.from_numpy(y.view(np.int32)))
        rc = lib.mp_exclusive_scan_noalloc(C.c_void_p(t.data_ptr()), C.c_void_p(t.data_ptr()), n,
                                           C.c_void_p(stream.cuda_stream))
        assert rc == _abi.MP_OK, lib.mp_last_error()
        torch.cuda.synchronize()
        out = t.cpu().numpy().view(np.uint32)
        np.testing.assert_array_equal(out, (np.cumsum(y, dtype=np.uint64) - y).astype(np.uint32))
        assert buf[:off].abs().sum().item() == 0  # nothing written before the array
