"""Snapshot byte layout (host side, no GPU): the Python mirror of
mtlphys_b200/csrc/snapshot.h matches the C++ structs, and round-trips."""
import ctypes as C
import os
import subprocess
import tempfile

import numpy as np
import pytest

from mtlphys_b200 import _abi, snapshot

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _cxx_layout():
    src = f"""
#include <cstdio>
#include <cstddef>
#include "{ROOT}/mtlphys_b200/csrc/snapshot.h"
using namespace mpb;
int main() {{
  std::printf("%zu %zu %zu %zu %zu %zu %zu\\n", sizeof(SnapshotHeader), sizeof(SnapshotScene),
              offsetof(SnapshotScene, desc), offsetof(SnapshotScene, scene_id),
              offsetof(SnapshotScene, count), offsetof(SnapshotScene, dt), offsetof(SnapshotScene, sphere));
  return 0;
}}"""
    with tempfile.TemporaryDirectory() as d:
        c, exe = os.path.join(d, "l.cpp"), os.path.join(d, "l")
        open(c, "w").write(src)
        subprocess.run(["g++", "-std=c++17", c, "-o", exe], check=True)
        return [int(x) for x in subprocess.run([exe], check=True, capture_output=True, text=True).stdout.split()]


def test_python_layout_matches_the_cxx_structs():
    S = snapshot.SceneRecord
    got = [C.sizeof(snapshot.Header), C.sizeof(S), S.desc.offset, S.scene_id.offset, S.count.offset,
           S.dt.offset, S.sphere.offset]
    assert _cxx_layout() == got


def make(n_per_scene=(3, 5), kind=snapshot.KIND_BATCH):
    rng = np.random.default_rng(1)
    scenes = []
    for i, n in enumerate(n_per_scene):
        r = snapshot.SceneRecord()
        r.params = _abi.default_params()
        r.params.scorr_k = 0.01 * (i + 1)
        r.desc = _abi.default_scene_desc()
        r.scene_id = i % 3
        r.count = n
        r.dt = 1.0 / 120.0
        for a in range(7):
            r.sphere[a] = a + i
        scenes.append(r)
    n = sum(n_per_scene)
    return snapshot.Snapshot(kind, scenes, rng.normal(size=(n, 4)).astype(np.float32),
                             rng.normal(size=(n, 4)).astype(np.float32))


def test_round_trip(tmp_path):
    s = make()
    p = tmp_path / "s.snap"
    snapshot.write(str(p), s)
    t = snapshot.read(str(p))
    assert t.kind == s.kind and t.particles == 8 and len(t.scenes) == 2
    np.testing.assert_array_equal(t.positions, s.positions)
    np.testing.assert_array_equal(t.velocities, s.velocities)
    assert bytes(t.scenes[1]) == bytes(s.scenes[1])
    assert abs(t.scenes[1].params.scorr_k - 0.02) < 1e-9
    assert len(snapshot.to_bytes(s)) == 64 + 2 * C.sizeof(snapshot.SceneRecord) + 32 * 8


def test_rejects_damaged_snapshots():
    data = snapshot.to_bytes(make())
    with pytest.raises(ValueError, match="magic"):
        snapshot.from_bytes(b"XXXXXXXX" + data[8:])
    with pytest.raises(ValueError, match="truncated"):
        snapshot.from_bytes(data[:-4])
    with pytest.raises(ValueError, match="header"):
        snapshot.from_bytes(data[:10])
    bad = bytearray(data)
    bad[8] = 9  # version
    with pytest.raises(ValueError, match="version"):
        snapshot.from_bytes(bytes(bad))
