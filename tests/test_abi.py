"""The C-ABI library loads and exports every symbol include/c3d.h declares."""
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "c3d.h")


def declared():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(c3d_[a-zA-Z0-9_]+)\s*\(", src)))


def test_library_builds_and_loads():
    from channel3d_parallel_b200 import _build, lib
    _build.build()
    assert lib.load() is not None


def test_exports_every_declared_symbol():
    from channel3d_parallel_b200 import lib
    so = lib.LIB_PATH
    out = subprocess.run(["nm", "-D", "--defined-only", so], capture_output=True, text=True).stdout
    exported = set(re.findall(r"\bT (c3d_\w+)", out))
    missing = [s for s in declared() if s not in exported]
    assert not missing, f"declared but not exported: {missing}"
    assert len(declared()) >= 39


def test_binding_covers_header():
    from channel3d_parallel_b200 import lib
    assert set(declared()) == set(lib.PROTOTYPES)


def test_no_device_error_is_loud():
    """Without a GPU, handle creation fails with C3D_ERR_NO_DEVICE (no CPU fallback)."""
    import channel3d_parallel_b200 as c3d
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except ImportError:
        pass
    with pytest.raises(c3d.C3DError) as e:
        c3d.Channel(nx_global=18, ny_global=17, nz_global=14, nu=1e-3, CFL=-1e-3)
    assert e.value.code == -7
