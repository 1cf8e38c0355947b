"""The C ABI library loads and exports every entry point include/gz_b200.h declares (no GPU
compute is started here)."""
import ctypes
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "gz_b200.h")


def declared():
    src = open(HEADER).read()
    return sorted(set(re.findall(r"^GZ_API\s+[\w\s\*]*?\b(gz_\w+)\s*\(", src, flags=re.M)))


def test_header_declares_the_surface():
    names = declared()
    for must in ("gz_create", "gz_destroy", "gz_apply_update_batch", "gz_ingest_records",
                 "gz_flush", "gz_connected_components", "gz_point_query", "gz_write_binary",
                 "gz_create_from_serialized", "gz_spanning_forest", "gz_last_query_rounds"):
        assert must in names


def test_library_exports_every_declared_symbol(gz):
    from graphzeppelin_b200 import _lib
    lib = _lib.load()
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.LIB_PATH], capture_output=True,
                         text=True, check=True).stdout
    exported = set(re.findall(r"\bT (gz_\w+)", out))
    names = declared()
    assert set(names) <= exported, set(names) - exported
    bound = {n for n, _, _ in _lib.SIGNATURES}
    assert set(names) == bound, set(names) ^ bound
    for n in names:
        assert getattr(lib, n) is not None


def test_status_strings(gz):
    from graphzeppelin_b200 import _lib
    assert _lib.status_string(0) == "ok"
    assert _lib.status_string(3) == "out of samples"
    assert _lib.status_string(4) == "updates locked"


def test_library_is_built_for_sm100a():
    from graphzeppelin_b200 import build
    assert "arch=compute_100a,code=sm_100a" in " ".join(build.ARCH)


def _has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.mark.skipif(_has_gpu(), reason="checks the no-GPU error path")
def test_no_device_fails_loudly(gz):
    with pytest.raises(gz.GZError) as e:
        gz.CCSketchAlg(16, 1)
    assert e.value.status == 10  # GZ_ERR_NO_DEVICE: there is no CPU fallback
