"""buildSpatialHash on the GPU (engine/src/Engine.cpp:601-679) through the C
ABI: the reference's own layouts (tests/test_spatial.cpp) against the golden
vectors of its shaders, and large random inputs bit-exact against the
oracle, including particles outside the box, NaN coordinates and cells past
the in-place ranking limit."""
import numpy as np
import pytest

from mtlphys_b200 import Engine, _abi
from oracle import oracle as O
from parity import assert_equal_u32, golden

pytestmark = pytest.mark.gpu
G = golden()
LAYOUTS = ["hash_points", "three_cells", "isolated", "close_pair", "lattice_099"]


@pytest.fixture(scope="module")
def eng(cuda):
    e = Engine(0)
    yield e
    e.close()


def run_hash(e, pos):
    e.reset(len(pos))
    e.set_positions(pos)
    e.build_spatial_hash()
    assert e.check_errors() == 0
    return e.cell_hashes(), e.cell_start(), e.sorted_index(), e.neighbor_counts()


@pytest.mark.parametrize("name", LAYOUTS)
def test_layouts_match_reference_shaders(eng, name):
    k = f"spatial/{name}/"
    h, cs, si, nc = run_hash(eng, G[k + "pos"])
    assert len(cs) == eng.total_cells() + 1 == 324001
    assert_equal_u32(h, G[k + "hashes"], "hashes")
    occ = np.nonzero(np.diff(cs))[0]
    assert_equal_u32(occ, G[k + "occupied_cells"], "occupied cells")
    assert_equal_u32(cs[occ], G[k + "occupied_start"], "cell starts")
    assert cs[-1] == len(h)
    assert_equal_u32(si, G[k + "sorted_index"], "sortedIndex")
    assert_equal_u32(nc, G[k + "neighbor_counts"], "neighbor counts")


def test_reference_known_answers(eng):
    assert (run_hash(eng, G["spatial/isolated/pos"])[3] == 0).all()
    assert list(run_hash(eng, G["spatial/close_pair/pos"])[3]) == [1, 1]
    nc = run_hash(eng, G["spatial/lattice_099/pos"])[3]
    assert nc[13] == 6 and nc[0] < nc[13] and nc[26] < nc[13]


def random_positions(n, seed, outside=0.02, nans=0):
    rng = np.random.default_rng(seed)
    lo = np.array([-3.0, -3.0, -3.0])
    hi = np.array([3.0, 6.0, 3.0])
    pos = np.ones((n, 4), np.float32)
    pos[:, :3] = rng.uniform(lo, hi, size=(n, 3))
    k = int(n * outside)
    pos[:k, :3] = rng.uniform(lo - 2, hi + 2, size=(k, 3))
    if nans:
        pos[k:k + nans, rng.integers(0, 3)] = np.nan
    rng.shuffle(pos)
    return pos


@pytest.mark.parametrize("n,seed", [(1_000_003, 1), (4097, 2)])
def test_random_hash_bit_exact(eng, n, seed):
    pos = random_positions(n, seed, nans=3)
    h, cs, si, nc = run_hash(eng, pos)
    oh, ocs, osi, onc = O.build_spatial_hash(_abi.default_params(), pos)
    assert_equal_u32(h, oh, "hashes")
    assert_equal_u32(cs, ocs, "cellStart")
    assert_equal_u32(si, osi, "sortedIndex")
    assert_equal_u32(nc, onc, "neighbor counts")


def test_dense_lattice_hash_bit_exact(eng):
    # rest packing: 8 particles per cell, ~30 neighbours each
    p = _abi.default_params()
    pos = O.seed_scene(p, _abi.MP_SCENE_DAM_BREAK, 400_000)
    h, cs, si, nc = run_hash(eng, pos)
    oh, ocs, osi, onc = O.build_spatial_hash(p, pos)
    assert_equal_u32(si, osi, "sortedIndex")
    assert_equal_u32(nc, onc, "neighbor counts")


@pytest.mark.parametrize("crowd", [257, 5000])
def test_crowded_cells_use_the_long_segment_path(eng, crowd):
    pos = random_positions(20_000, 7)
    rng = np.random.default_rng(crowd)
    idx = rng.choice(len(pos), size=crowd, replace=False)
    pos[idx, :3] = [0.0512, 0.0123, -1.0345]  # all in one cell (and all at one point)
    h, cs, si, nc = run_hash(eng, pos)
    oh, ocs, osi, onc = O.build_spatial_hash(_abi.default_params(), pos)
    assert_equal_u32(si, osi, "sortedIndex")
    assert_equal_u32(nc, onc, "neighbor counts")
    c = oh[idx[0]]
    assert ocs[c + 1] - ocs[c] >= crowd


def test_hash_is_deterministic(eng):
    pos = random_positions(300_000, 9)
    a = run_hash(eng, pos)
    b = run_hash(eng, pos)
    for x, y in zip(a, b):
        assert np.array_equal(x, y)
