"""Bounds-checked build (CPU): the checked library reports itself, keeps a
region list whose containment rule is exact at the edges, and the default
build compiles the checks away (its region calls answer NOT_SUPPORTED)."""
import ctypes as C
import os

import pytest

from hicma_parsec_b200 import build, tlr


def _load(path):
    if not os.path.exists(path):
        pytest.skip("library not built")
    lib = C.CDLL(path)
    lib.hicma_tlr_bounds_checked.restype = C.c_int
    lib.hicma_tlr_bounds_register.argtypes = [C.c_void_p, C.c_size_t]
    lib.hicma_tlr_bounds_unregister.argtypes = [C.c_void_p]
    lib.hicma_tlr_bounds_inside.argtypes = [C.c_void_p, C.c_size_t]
    return lib


def test_checked_build_region_rule():
    lib = _load(build.LIB_CHECKED)
    assert lib.hicma_tlr_bounds_checked() == 1
    base = 0x7F0000001000                # an address value only: the list is never dereferenced
    assert lib.hicma_tlr_bounds_inside(base, 8) == 0
    assert lib.hicma_tlr_bounds_register(base, 4096) == 0
    assert lib.hicma_tlr_bounds_inside(base, 4096) == 1
    assert lib.hicma_tlr_bounds_inside(base + 4088, 8) == 1
    assert lib.hicma_tlr_bounds_inside(base + 4089, 8) == 0       # one byte past the end
    assert lib.hicma_tlr_bounds_inside(base - 8, 16) == 0         # starts before the region
    assert lib.hicma_tlr_bounds_inside(base + 100, 0) == 1        # empty extents always pass
    # a second region next to the first: an extent across both is not inside one region
    assert lib.hicma_tlr_bounds_register(base + 4096, 4096) == 0
    assert lib.hicma_tlr_bounds_inside(base + 4000, 200) == 0
    assert lib.hicma_tlr_bounds_inside(base + 5000, 200) == 1
    assert lib.hicma_tlr_bounds_unregister(base + 4096) == 0
    assert lib.hicma_tlr_bounds_inside(base + 5000, 200) == 0
    assert lib.hicma_tlr_bounds_unregister(base) == 0
    assert lib.hicma_tlr_bounds_inside(base, 8) == 0
    assert lib.hicma_tlr_bounds_register(None, 8) == tlr.ERR_ARG


def test_default_build_has_no_checks():
    lib = _load(build.LIB)
    assert lib.hicma_tlr_bounds_checked() == 0
    assert lib.hicma_tlr_bounds_register(0x1000, 8) == tlr.ERR_NOT_SUPPORTED
    assert lib.hicma_tlr_bounds_inside(0x1000, 8) == tlr.ERR_NOT_SUPPORTED


def test_loader_selects_the_checked_build(monkeypatch):
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    code = "from hicma_parsec_b200 import tlr; print(tlr.load_library().hicma_tlr_bounds_checked())"
    for env, want in (("checked", "1"), ("", "0")):
        r = subprocess.run([sys.executable, "-c", code], cwd=root, capture_output=True, text=True, timeout=120,
                           env={**os.environ, "HICMA_TLR_LIB": env})
        assert r.returncode == 0, r.stderr
        assert r.stdout.strip() == want


def test_missing_library_fails_loudly():
    """No CPU fallback: without the CUDA library the binding refuses to load."""
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    code = ("from hicma_parsec_b200 import tlr\n"
            "try:\n    tlr.load_library()\nexcept RuntimeError as e:\n    print('refused:', e)\n")
    r = subprocess.run([sys.executable, "-c", code], cwd=root, capture_output=True, text=True, timeout=120,
                       env={**os.environ, "HICMA_TLR_LIB": os.path.join(root, "no_such_lib.so")})
    assert r.returncode == 0 and r.stdout.startswith("refused:") and "not built" in r.stdout
