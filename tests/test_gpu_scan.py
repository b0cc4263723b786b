"""mp_exclusive_scan (runExclusiveScan, engine/src/Engine.cpp:843-882) on the
GPU against the exclusive prefix sum, over the reference's test cases
(tests/test_scan.cpp) plus sizes past its 1024^2 cap, ragged tails,
unaligned pointers, in-place use and 2^32 wraparound."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def np_excl(x):
    x = np.asarray(x, np.uint32)
    return (np.cumsum(x, dtype=np.uint64) - x).astype(np.uint32)


def rand(n, seed, maxval):
    return np.random.RandomState(seed).randint(0, maxval + 1, size=n).astype(np.uint32)


CASES = {
    "zeros_100": lambda: np.zeros(100, np.uint32),
    "ones_500": lambda: np.ones(500, np.uint32),
    "rand_1024": lambda: rand(1024, 0xA, 7),
    "rand_700": lambda: rand(700, 0xB, 7),
    "rand_2048": lambda: rand(2048, 0xC, 7),
    "rand_635626": lambda: rand(635626, 0xD, 3),
    "one": lambda: np.array([7], np.uint32),
    "tile_4096": lambda: rand(4096, 1, 9),
    "tile_4097": lambda: rand(4097, 2, 9),
    "past_ref_cap_3M": lambda: rand(3_000_001, 3, 5),
    "wrap_u32_1M": lambda: np.random.RandomState(4).randint(0, 2**32, size=1_000_003,
                                                            dtype=np.uint64).astype(np.uint32),
}


def gpu_scan(x, in_place=False, offset=0):
    import torch

    from mtlphys_b200 import exclusive_scan

    buf = torch.zeros(len(x) + offset, dtype=torch.int32, device="cuda")
    t = buf[offset:]
    t.copy_(torch.from_numpy(x.view(np.int32)))
    out = t if in_place else torch.full_like(t, -1)
    exclusive_scan(t, out)
    torch.cuda.synchronize()
    return out.cpu().numpy().view(np.uint32)


@pytest.mark.parametrize("name", sorted(CASES))
def test_scan_matches_prefix_sum(cuda, name):
    x = CASES[name]()
    got = gpu_scan(x)
    want = np_excl(x)
    bad = np.nonzero(got != want)[0]
    assert bad.size == 0, f"first mismatch at {bad[0]}: got {got[bad[0]]} want {want[bad[0]]}"


def test_scan_in_place(cuda):
    x = rand(100_003, 5, 7)
    np.testing.assert_array_equal(gpu_scan(x, in_place=True), np_excl(x))


@pytest.mark.parametrize("offset", [1, 2, 3])
def test_scan_unaligned_pointers(cuda, offset):
    x = rand(50_001, 6 + offset, 7)
    np.testing.assert_array_equal(gpu_scan(x, offset=offset), np_excl(x))


def test_scan_rejects_small_scratch(cuda):
    import ctypes as C

    import torch

    from mtlphys_b200 import _abi

    lib = _abi.load()
    t = torch.zeros(10_000, dtype=torch.int32, device="cuda")
    scratch = torch.zeros(8, dtype=torch.uint8, device="cuda")
    rc = lib.mp_exclusive_scan(C.c_void_p(t.data_ptr()), C.c_void_p(t.data_ptr()), 10_000,
                               C.c_void_p(scratch.data_ptr()), 8, None)
    assert rc == _abi.MP_ERR_INVALID_ARGUMENT
    assert lib.mp_exclusive_scan(None, None, 0, None, 0, None) == _abi.MP_OK  # n == 0 no-op
