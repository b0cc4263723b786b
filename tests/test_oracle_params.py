"""The oracle's own parameter structs and workloads (oracle/params.py, which
the checker and the benchmark's reference arm use so that they never load
the product library) equal the product's: struct layouts, the reference
defaults that mp_default_params() returns, the lattice rest density and the
benchmark workloads, byte for byte.  Runs without a GPU (the product library
loads on the host for its pure host functions)."""
import ctypes as C

import pytest

from mtlphys_b200 import _abi, configs
from oracle import params as P


@pytest.mark.parametrize("ours,theirs", [(P.PBFParams, _abi.PBFParams), (P.SceneDesc, _abi.SceneDesc)])
def test_layouts_equal(ours, theirs):
    assert C.sizeof(ours) == C.sizeof(theirs)
    assert [(f, getattr(ours, f).offset) for f, _ in ours._fields_] == \
           [(f, getattr(theirs, f).offset) for f, _ in theirs._fields_]


def test_defaults_equal_mp_default_params():
    assert bytes(P.default_params()) == bytes(_abi.default_params())
    assert bytes(P.default_scene_desc()) == bytes(_abi.default_scene_desc())


def test_rest_density_equals_the_library():
    lib = _abi.load()
    for h, sp in ((0.1, 0.05), (0.1, 0.035), (0.2, 0.1), (0.05, 0.02)):
        assert P.lattice_rest_density(h, sp) == lib.mp_lattice_rest_density(h, sp)


@pytest.mark.parametrize("name", sorted(P.WORKLOADS))
def test_workloads_equal(name):
    a, b = P.WORKLOADS[name](), configs.WORKLOADS[name]()
    assert bytes(a.params) == bytes(b.params)
    assert bytes(a.desc) == bytes(b.desc)
    assert (a.name, a.scene, a.n, a.dt, a.steps) == (b.name, b.scene, b.n, b.dt, b.steps)
    assert a.describe() == b.describe()


def test_product_structs_are_accepted_by_the_oracle():
    from oracle import oracle as O

    w = configs.cube_drop(side=6)
    a = O.seed_scene(w.params, w.scene, w.n, w.desc)
    wo = P.cube_drop(side=6)
    b = O.seed_scene(wo.params, wo.scene, wo.n, wo.desc)
    assert (a == b).all()
