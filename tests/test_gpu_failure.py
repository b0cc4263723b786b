"""Failure paths on the GPU, none of which faults or hangs it.

The reference aborts the process when something goes wrong
(engine/src/Engine.cpp:72-83, 407-413, 849-854) and creates its buffers
without checking (Engine.cpp:390-395).  This engine reports instead:
- every device-side wait is bounded.  A test lowers the bound
  (mp_set_spin_limit) and makes the wait run out: a scan whose look-back
  waits for descriptors that no tile writes, a batch whose grid barrier waits
  for a block that does not exist.  The status comes back as
  MP_ERR_SPIN_LIMIT within milliseconds, the outputs stay inside their
  buffers, and the handle works again afterwards;
- device allocations go through an injectable allocator.  One that refuses
  makes reset return MP_ERR_OUT_OF_MEMORY and leaves the engine or batch
  empty but usable: with memory available again it resets and steps exactly
  like a fresh one."""
import ctypes as C
import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SHORT = 2000  # polls: a wait of ~0.1-2 ms


def _lib():
    from mtlphys_b200 import _abi

    return _abi.load()


@pytest.fixture
def short_waits(cuda):
    lib = _lib()
    lib.mp_set_spin_limit(SHORT)
    yield lib
    lib.mp_set_spin_limit(0)


def np_excl(x):
    return (np.cumsum(x, dtype=np.uint64) - x).astype(np.uint32)


def test_scan_lookback_that_runs_out_is_reported(short_waits):
    import torch

    from mtlphys_b200 import _abi

    lib = short_waits
    tile = 4096
    tiles = 6
    n = (tiles - 1) * tile + 1000
    x = np.random.default_rng(7).integers(0, 9, n).astype(np.uint32)
    t = torch.from_numpy(x.view(np.int32)).cuda()
    out = torch.full_like(t, -1)
    nbytes = int(lib.mp_exclusive_scan_scratch_bytes(n))
    scratch = torch.zeros(nbytes, dtype=torch.uint8, device="cuda")
    stream = torch.cuda.current_stream()
    sh = C.c_void_p(stream.cuda_stream)
    t0 = time.perf_counter()
    # the ticket starts one short of a whole epoch: the first tile launched is
    # the last tile, of the old epoch, and its predecessors all belong to the next
    rc = lib.mp_debug_exclusive_scan_from_ticket(C.c_void_p(t.data_ptr()), C.c_void_p(out.data_ptr()), n,
                                                 C.c_void_p(scratch.data_ptr()), nbytes, tiles - 1, sh)
    assert rc == _abi.MP_OK, lib.mp_last_error()
    rc = lib.mp_exclusive_scan_status(C.c_void_p(scratch.data_ptr()), sh)
    elapsed = time.perf_counter() - t0
    assert rc == _abi.MP_ERR_SPIN_LIMIT, lib.mp_last_error()
    assert b"look-back" in lib.mp_last_error()
    assert elapsed < 5.0
    got = out.cpu().numpy().view(np.uint32)
    want = np_excl(x)
    last = (tiles - 1) * tile
    # the other tiles are right; the last one has only its own prefix
    np.testing.assert_array_equal(got[:last], want[:last])
    np.testing.assert_array_equal(got[last:], want[last:] - want[last])
    # the status was cleared, and the same scratch serves a normal scan
    assert lib.mp_exclusive_scan_status(C.c_void_p(scratch.data_ptr()), sh) == _abi.MP_OK
    rc = lib.mp_exclusive_scan(C.c_void_p(t.data_ptr()), C.c_void_p(out.data_ptr()), n,
                               C.c_void_p(scratch.data_ptr()), nbytes, sh)
    assert rc == _abi.MP_OK
    assert lib.mp_exclusive_scan_status(C.c_void_p(scratch.data_ptr()), sh) == _abi.MP_OK
    np.testing.assert_array_equal(out.cpu().numpy().view(np.uint32), want)


def test_scan_status_of_a_completed_scan_is_ok(cuda):
    import torch

    from mtlphys_b200 import _abi

    lib = _lib()
    x = np.arange(100_000, dtype=np.uint32) % 5
    t = torch.from_numpy(x.view(np.int32)).cuda()
    out = torch.empty_like(t)
    sh = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    assert lib.mp_exclusive_scan_noalloc(C.c_void_p(t.data_ptr()), C.c_void_p(out.data_ptr()), len(x),
                                         sh) == _abi.MP_OK
    assert lib.mp_exclusive_scan_status(None, sh) == _abi.MP_OK
    np.testing.assert_array_equal(out.cpu().numpy().view(np.uint32), np_excl(x))


def _small_batch():
    from mtlphys_b200 import configs
    from mtlphys_b200.batch import Batch

    w = configs.batch_cubes(num=3, lo=2000, hi=6000)
    b = Batch(0)
    b.reset(w.counts, w.params, w.dts, w.scenes, w.descs)
    return b, w


@pytest.mark.parametrize("graph", [False, True])
def test_batch_barrier_that_runs_out_aborts_the_step_and_rearms(short_waits, graph):
    from mtlphys_b200 import _abi

    lib = short_waits
    b, w = _small_batch()
    try:
        b.set_graph_mode(graph)
        b.step()
        assert b.check_errors() == 0
        saved = b.snapshot_bytes()
        assert lib.mp_batch_debug_barrier_extra(b._h, 1) == _abi.MP_OK
        t0 = time.perf_counter()
        b.step()
        b.step()  # does nothing: the batch stays stopped until its error is read
        bits = C.c_uint32()
        rc = lib.mp_batch_check_errors(b._h, C.byref(bits))
        assert time.perf_counter() - t0 < 10.0
        assert rc == _abi.MP_ERR_SPIN_LIMIT and bits.value & _abi.MP_DEVERR_SPIN_LIMIT
        # re-armed: the same batch, restored, steps exactly like a fresh one
        assert lib.mp_batch_debug_barrier_extra(b._h, 0) == _abi.MP_OK
        b.restore_bytes(saved)
        for _ in range(3):
            b.step()
        assert b.check_errors() == 0
        ref, _ = _small_batch()
        try:
            for _ in range(4):
                ref.step()
            assert ref.check_errors() == 0
            np.testing.assert_array_equal(b.positions(), ref.positions())
            np.testing.assert_array_equal(b.velocities(), ref.velocities())
        finally:
            ref.close()
    finally:
        b.close()


class RefusingAllocator:
    """A device allocator (torch's caching allocator underneath) that refuses
    every request once `refuse` is set, and counts what it hands out."""

    def __init__(self):
        import torch

        from mtlphys_b200 import _abi

        self.refuse = False
        self.refused = 0
        self.live = {}

        def alloc(pp, nbytes, device, user):
            if self.refuse:
                self.refused += 1
                return 1
            ptr = torch.cuda.caching_allocator_alloc(int(nbytes), int(device))
            self.live[int(ptr)] = int(nbytes)
            pp[0] = ptr
            return 0

        def free(ptr, device, user):
            self.live.pop(int(ptr))
            torch.cuda.caching_allocator_delete(int(ptr))

        self._alloc = _abi.DEVICE_ALLOC_FN(alloc)
        self._free = _abi.DEVICE_FREE_FN(free)

    def install(self):
        assert _lib().mp_set_device_allocator(C.cast(self._alloc, C.c_void_p),
                                              C.cast(self._free, C.c_void_p), None) == 0

    @staticmethod
    def uninstall():
        assert _lib().mp_set_device_allocator(None, None, None) == 0


def test_engine_reset_out_of_memory_leaves_it_empty_and_usable(cuda):
    from mtlphys_b200 import Engine, MPError, _abi, configs

    w = configs.cube_drop(side=16)
    a = RefusingAllocator()
    e = Engine(0)
    try:
        e.set_params(w.params)
        e.reset(1000, w.scene)
        a.install()
        a.refuse = True
        with pytest.raises(MPError) as ex:
            e.reset(w.n, w.scene, w.desc)  # needs larger particle buffers
        assert ex.value.code == _abi.MP_ERR_OUT_OF_MEMORY and a.refused >= 1
        assert e.particle_count() == 0
        e.step(w.dt)  # an empty engine steps as a no-op
        e.build_spatial_hash()
        assert e.check_errors() == 0
        a.refuse = False
        e.reset(w.n, w.scene, w.desc)  # through the caller's allocator now
        assert a.live, "the reset did not allocate through the installed allocator"
        for _ in range(4):
            e.step(w.dt)
        assert e.check_errors() == 0
        got = e.positions()
    finally:
        a.uninstall()
        e.close()
    assert not a.live, "blocks were not given back to the allocator that made them"
    ref = Engine(0)
    try:
        ref.set_params(w.params)
        ref.reset(w.n, w.scene, w.desc)
        for _ in range(4):
            ref.step(w.dt)
        np.testing.assert_array_equal(got, ref.positions())
    finally:
        ref.close()


def test_batch_reset_out_of_memory_leaves_it_empty_and_usable(cuda):
    from mtlphys_b200 import MPError, _abi, configs
    from mtlphys_b200.batch import Batch

    w = configs.batch_cubes(num=4, lo=2000, hi=5000)
    a = RefusingAllocator()
    b = Batch(0)
    try:
        a.install()
        a.refuse = True
        with pytest.raises(MPError) as ex:
            b.reset(w.counts, w.params, w.dts, w.scenes, w.descs)
        assert ex.value.code == _abi.MP_ERR_OUT_OF_MEMORY
        assert b.particle_count() == 0 and b.scene_count() == 0
        b.step()
        assert b.check_errors() == 0
        a.refuse = False
        b.reset(w.counts, w.params, w.dts, w.scenes, w.descs)
        for _ in range(3):
            b.step()
        assert b.check_errors() == 0
        got = b.positions()
    finally:
        a.uninstall()
        b.close()
    assert not a.live
    ref = Batch(0)
    try:
        ref.reset(w.counts, w.params, w.dts, w.scenes, w.descs)
        for _ in range(3):
            ref.step()
        np.testing.assert_array_equal(got, ref.positions())
    finally:
        ref.close()
