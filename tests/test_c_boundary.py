"""The C boundary compiled as C: a program written against include/monolis.h
(tests/c/solver_c.c), built with gcc and linked against the oracle (here)
and against the product library (on the GPU), and the struct layout and
constant values of include/monolis.h against those of the reference's own
headers (tests/c/abi_layout.c; fixture tests/golden/abi_layout_reference.txt,
written by tests/golden/make_abi_layout.py from the reference tree)."""
import os
import subprocess

import pytest

from monolis_b200 import api

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
INC = os.path.join(ROOT, "include")
CDIR = os.path.join(ROOT, "tests", "c")


def _build(tmp_path, src, lib=None):
    exe = str(tmp_path / os.path.splitext(os.path.basename(src))[0])
    cmd = ["gcc", "-std=c11", "-Wall", "-Wextra", "-Werror", "-I", INC, os.path.join(CDIR, src)]
    if lib:
        cmd += [lib, f"-Wl,-rpath,{os.path.dirname(lib)}", "-lm"]
    subprocess.run(cmd + ["-o", exe], check=True, capture_output=True, text=True)
    return exe


def test_struct_layout_and_constants_match_reference_headers(tmp_path):
    exe = _build(tmp_path, "abi_layout.c")
    ours = subprocess.run([exe], check=True, capture_output=True, text=True).stdout.splitlines()
    with open(os.path.join(ROOT, "tests", "golden", "abi_layout_reference.txt")) as f:
        ref = f.read().splitlines()
    assert len(ref) == 90
    assert ours == ref


def test_c_program_against_oracle(tmp_path, oracle):
    exe = _build(tmp_path, "solver_c.c", oracle.path)
    out = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stdout + out.stderr
    assert out.stdout.strip().endswith("all ok")


@pytest.mark.gpu
def test_c_program_against_product(tmp_path, gpu):
    exe = _build(tmp_path, "solver_c.c", api.PRODUCT_SO)
    out = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stdout + out.stderr
    assert out.stdout.strip().endswith("all ok")
    cases = [ln for ln in out.stdout.splitlines() if ln.startswith("ndof")]
    assert len(cases) == 6 and all(ln.endswith(" ok") for ln in cases)
