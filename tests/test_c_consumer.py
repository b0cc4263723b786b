"""A compiled C consumer of the C ABI (tests/c_consumer.c): the header
compiles as strict C99, the program links against the product library like
the reference's Obj-C++ bridge links the engine (app/bridge/EngineBridge.mm),
and, on a GPU, runs create -> reset -> step -> download, the hash invariants
and a scan through nothing but the header's declarations."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.join(ROOT, "mtlphys_b200")


def build(tmp_path) -> str:
    exe = str(tmp_path / "c_consumer")
    subprocess.run(["gcc", "-std=c99", "-Wall", "-Wextra", "-Werror", "-pedantic", "-O1",
                    "-I", os.path.join(ROOT, "include"), os.path.join(ROOT, "tests", "c_consumer.c"),
                    "-L", LIBDIR, "-lmtlphys_b200", f"-Wl,-rpath,{LIBDIR}", "-lm", "-o", exe],
                   check=True, capture_output=True, text=True)
    return exe


def test_c_consumer_builds_and_runs_host_calls(tmp_path):
    exe = build(tmp_path)
    out = subprocess.run([exe, "abi"], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stderr
    assert "ok abi" in out.stdout


@pytest.mark.gpu
def test_c_consumer_steps_the_engine(tmp_path, cuda):
    exe = build(tmp_path)
    out = subprocess.run([exe, "run"], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stdout + out.stderr
    for line in ("ok isolated", "ok cube_drop", "ok scan", "ok all"):
        assert line in out.stdout, out.stdout
