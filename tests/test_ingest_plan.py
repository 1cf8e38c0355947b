"""The host-record ingest chunk plan (graphzeppelin_b200/csrc/gz_ingest_plan.h), compiled with g++
and checked over 2000+ call lengths on the CPU: the chunks tile each call exactly and fit the
staging buffers, and the shaped form (doubling first chunks, a wave per chunk, then a tail of
halving chunks folded by one wave at the next flush) is taken exactly when it applies."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_ingest_plan_properties(tmp_path):
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("g++ not found")
    exe = str(tmp_path / "ingest_plan_test")
    subprocess.run([gxx, "-std=c++14", "-O1", "-Wall", "-Werror",
                    "-I", os.path.join(ROOT, "graphzeppelin_b200", "csrc"),
                    os.path.join(ROOT, "tests", "cpp", "ingest_plan_test.cpp"), "-o", exe],
                   check=True, capture_output=True, text=True)
    out = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stdout + out.stderr
    assert "ingest plan ok" in out.stdout
    # the dense 1.4e8-record stream: 8 Mi first, full 16 Mi chunks, a tail of 8, 4 and 2 Mi
    plan = out.stdout.split("dense plan:")[1].split("(")[0].split()
    assert plan[0] == "8.00" and plan[1] == "16.00" and plan[-3:] == ["8.00", "4.00", "2.00"]
