"""The header-only C++ facade (include/gz_b200.hpp) compiles, and on a GPU a C++ program using
it reproduces the reference tests' known answers through libgz_b200.so."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cpp", "facade_test.cpp")


def _compile(out):
    from graphzeppelin_b200 import _lib
    _lib.load()
    gxx = shutil.which("g++")
    cmd = [gxx, "-std=c++14", "-O1", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"), SRC,
           "-o", out, "-L", os.path.dirname(_lib.LIB_PATH), "-lgz_b200",
           "-Wl,-rpath," + os.path.dirname(_lib.LIB_PATH)]
    subprocess.run(cmd, check=True, capture_output=True, text=True)


def test_facade_compiles(tmp_path):
    _compile(str(tmp_path / "facade_test"))


@pytest.mark.gpu
def test_facade_reproduces_reference_answers(tmp_path):
    from _golden import GOLDEN
    exe = str(tmp_path / "facade_test")
    _compile(exe)
    out = subprocess.run([exe, os.path.join(GOLDEN, "mult_v1024.gzs"), str(tmp_path / "ck.bin")],
                         capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stdout + out.stderr
    assert "facade ok: 78 components" in out.stdout
