"""CPU tests of the C-ABI boundary: the library builds for sm_100a, loads,
and exports every entry point that include/*.h declares. No compute calls."""
import ctypes
import glob
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = []
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        for m in re.finditer(r"^\s*(?:const\s+)?\w+\s*\*?\s*(sf_\w+)\s*\(", src, flags=re.M):
            names.append(m.group(1))
    return sorted(set(names))


def test_header_declares_entry_points():
    names = declared_functions()
    assert "sf_create" in names and "sf_step" in names and "sf_step_linear" in names
    assert len(names) >= 20


def test_library_exports_every_declared_symbol():
    from stratiflow_b200 import build
    lib_path = build.build()
    lib = ctypes.CDLL(lib_path)
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_python_binding_covers_header():
    import stratiflow_b200 as sf
    assert sorted(sf.EXPORTS) == declared_functions()


def test_package_fails_loudly_without_library(tmp_path):
    import stratiflow_b200 as sf
    saved = sf._lib
    sf._lib = None
    try:
        with pytest.raises(sf.SFError):
            sf.load_library(str(tmp_path / "missing.so"))
    finally:
        sf._lib = saved


def test_library_is_built_for_sm100a():
    from stratiflow_b200 import build
    assert "arch=compute_100a,code=sm_100a" in " ".join(build.ARCH)


def host_functions():
    src = open(os.path.join(ROOT, "stratiflow_b200", "host", "sf_host.cpp")).read()
    return sorted(set(re.findall(r"^(?:int|const char\*)\s+(sfh_\w+)\s*\(", src, flags=re.M)))


def test_host_library_exports_its_entry_points_and_python_binds_them():
    """libstratiflow_host.so (the C++ drivers) exports every entry point
    sf_host.cpp defines, and the Python front end gives each of them its
    argument types (ctypes would otherwise pass doubles as ints)."""
    from stratiflow_b200 import build, drivers
    build.build()
    names = host_functions()
    assert {"sfh_newton_fixed", "sfh_arnoldi", "sfh_inverse_iteration", "sfh_critical_point",
            "sfh_find_hopf", "sfh_linear_evolve"} <= set(names)
    L = drivers.load_host()
    for n in names:
        assert hasattr(L, n), n
        if n != "sfh_last_error":
            assert getattr(L, n).argtypes is not None, n
