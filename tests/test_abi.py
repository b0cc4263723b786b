"""The C ABI library loads without a GPU, exports every function the header
declares, and its struct layouts match the ctypes mirror.  No compute calls."""
import ctypes as C
import os
import re
import subprocess
import tempfile

import pytest

from mtlphys_b200 import _abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "mtlphys_b200.h")


def header_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(mp_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_the_engine_surface():
    names = header_functions()
    for must in ("mp_engine_create", "mp_engine_reset", "mp_engine_reset_scene", "mp_engine_step",
                 "mp_engine_build_spatial_hash", "mp_engine_particle_count",
                 "mp_engine_total_cells", "mp_engine_cell_size", "mp_engine_current_scene",
                 "mp_exclusive_scan", "mp_engine_set_params"):
        assert must in names


def test_library_exports_every_declared_symbol():
    lib = _abi.load()
    missing = [n for n in header_functions() if not hasattr(lib, n)]
    assert not missing, f"not exported: {missing}"
    # and the ctypes prototypes cover the header
    assert set(header_functions()) <= set(_abi.PROTOTYPES), set(header_functions()) - set(_abi.PROTOTYPES)


def _c_layout(struct: str, fields):
    src = ["#include <stdio.h>", "#include <stddef.h>", f'#include "{HEADER}"', "int main(void){",
           f'printf("%zu\\n", sizeof({struct}));']
    for f in fields:
        src.append(f'printf("%zu\\n", offsetof({struct}, {f}));')
    src.append("return 0;}")
    with tempfile.TemporaryDirectory() as d:
        c = os.path.join(d, "l.c")
        exe = os.path.join(d, "l")
        open(c, "w").write("\n".join(src))
        subprocess.run(["gcc", c, "-o", exe], check=True)
        out = subprocess.run([exe], check=True, capture_output=True, text=True).stdout.split()
    return [int(x) for x in out]


@pytest.mark.parametrize("cls,cname", [(_abi.PBFParams, "mp_pbf_params"), (_abi.SceneDesc, "mp_scene_desc")])
def test_struct_layout_matches_header(cls, cname):
    fields = [f for f, _ in cls._fields_]
    got = [C.sizeof(cls)] + [getattr(cls, f).offset for f in fields]
    assert _c_layout(cname, fields) == got


def test_default_params_are_the_reference_tunables():
    p = _abi.default_params()
    assert p.size == C.sizeof(_abi.PBFParams)
    assert p.solver_iterations == 5                      # Engine.cpp:39
    assert p.h == pytest.approx(0.10) and p.cell_size == pytest.approx(0.10)
    assert p.rest_density == 8000.0 and p.epsilon == 800.0
    assert p.damping == pytest.approx(0.996)
    assert list(p.gravity) == pytest.approx([0, -9.81, 0])
    assert list(p.bounds_min) == [-3, -3, -3] and list(p.bounds_max) == [3, 6, 3]
    assert p.scorr_k == pytest.approx(1e-4) and p.scorr_n == 4
    assert p.scorr_dq == pytest.approx(0.2) and p.max_delta == pytest.approx(0.3)
    assert p.foam_max_neighbors == 96.0


def test_lattice_rest_density():
    # 1 + 6 + 12 + 8 lattice sites inside h at spacing h/2: 5.15625 * W(0)
    rho = _abi.load().mp_lattice_rest_density(0.1, 0.05)
    assert rho == pytest.approx(8078.2013, abs=1e-3)


def test_last_error_starts_empty_and_null_args_are_rejected():
    lib = _abi.load()
    assert lib.mp_default_params(None) == _abi.MP_ERR_INVALID_ARGUMENT
    assert b"NULL" in lib.mp_last_error()
    assert lib.mp_engine_destroy(None) == _abi.MP_OK


def test_failure_hooks_are_host_calls():
    """mp_set_spin_limit and mp_set_device_allocator need no GPU; an
    allocator without a free function is refused."""
    lib = _abi.load()
    assert lib.mp_set_spin_limit(1000) == _abi.MP_OK
    assert lib.mp_set_spin_limit(0) == _abi.MP_OK
    alloc = _abi.DEVICE_ALLOC_FN(lambda pp, n, dev, user: 1)
    assert lib.mp_set_device_allocator(C.cast(alloc, C.c_void_p), None, None) == _abi.MP_ERR_INVALID_ARGUMENT
    assert lib.mp_set_device_allocator(None, None, None) == _abi.MP_OK
