"""The bounds-checked flavour of the library (-DCRITMC_CHECK) builds and exports
its report; a release build answers that it is not checked."""

from __future__ import annotations

import ctypes

from critmc_b200 import _build, _lib


def test_release_build_reports_not_checked():
    assert _lib.lib().critmc_check_report(None, 0) == -1


def test_checked_flavour_builds_and_exports_the_abi():
    path = _build.build(check=True)
    assert path.name == "libcritmc_b200_check.so"
    lib = ctypes.CDLL(str(path))
    for name in _lib.SIGNATURES:
        assert hasattr(lib, name), name
