"""The C-ABI library loads and exports every function include/galaxy_b200.h declares
(no compute calls: this runs without a GPU)."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    src = open(os.path.join(ROOT, "include", "galaxy_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(gs_[a-z0-9_]+)\s*\(", src)))


def test_header_declares_the_surface():
    names = declared_functions()
    for must in ["gs_create", "gs_destroy", "gs_update_params", "gs_apply_permutation",
                 "gs_upload_tree", "gs_refresh", "gs_step", "gs_star_formation",
                 "gs_read_positions", "gs_sort_build", "gs_run", "gs_get_tree",
                 "gs_morton_codes", "gs_radix_sort_indices", "gs_tree_build", "gs_sort_and_build",
                 "gs_energy", "gs_last_error"]:
        assert must in names


def test_library_exports_every_declared_symbol():
    from galaxy_sim_b200 import _lib, build

    build.build()
    L = ctypes.CDLL(_lib.LIB_PATH)
    missing = [n for n in declared_functions() if not hasattr(L, n)]
    assert not missing, missing
    bound = {name for name, _, _ in _lib.SIGNATURES}
    assert set(declared_functions()) <= bound


def test_library_reports_errors_without_gpu():
    from galaxy_sim_b200 import _lib

    L = _lib.lib()
    assert L.gs_version().startswith(b"galaxy_b200")
    h = ctypes.c_void_p()
    assert L.gs_create(0, None, None, ctypes.byref(h)) == _lib.GS_EINVAL
    assert b"N must be" in L.gs_last_error(None)
    assert L.gs_step(None) == _lib.GS_EINVAL


def test_fault_injection_settings_check_their_arguments_without_gpu():
    """The host-side failure-detection settings are armed and disarmed on the
    host alone, and refuse values that mean nothing."""
    from galaxy_sim_b200 import _lib

    L = _lib.lib()
    assert L.gs_test_fail_alloc(-2) == _lib.GS_EINVAL
    assert b"allocation count or -1" in L.gs_last_error(None)
    assert L.gs_test_fail_alloc(7) == _lib.GS_OK
    assert L.gs_test_fail_alloc(-1) == _lib.GS_OK
    assert L.gs_test_sort_lookback(0, -1) == _lib.GS_EINVAL
    assert b"spin_limit must be positive" in L.gs_last_error(None)
    assert L.gs_test_sort_lookback(1 << 20, -2) == _lib.GS_EINVAL
    assert L.gs_test_sort_lookback(1 << 20, -1) == _lib.GS_OK


def test_missing_library_fails_loudly(monkeypatch, tmp_path):
    from galaxy_sim_b200 import _lib

    monkeypatch.setattr(_lib, "_lib", None)
    monkeypatch.setattr(_lib, "LIB_PATH", str(tmp_path / "absent.so"))
    with pytest.raises(ImportError):
        _lib.lib()
