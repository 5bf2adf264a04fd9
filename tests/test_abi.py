"""The C-ABI library loads and exports every entry point declared in
include/fcfd.h (no compute calls; CPU only)."""
import ctypes
import os
import re

from tests.conftest import ROOT


def _declared():
    text = open(os.path.join(ROOT, "include", "fcfd.h")).read()
    return sorted(set(re.findall(r"\b(fcfd_[a-z0-9_]+)\s*\(", text)))


def test_header_symbols_exported(fb):
    lib = ctypes.CDLL(fb.LIB_PATH)
    missing = [s for s in _declared() if not hasattr(lib, s)]
    assert not missing, missing


def test_version_and_error_strings(fb):
    assert b"sm_100a" in fb.lib.fcfd_version()
    assert isinstance(fb.lib.fcfd_last_error(), bytes)


def test_bad_deck_returns_status(fb, tmp_path):
    """A missing deck is an ERR_INPUT status, not an exit (reference: exit(1))."""
    import pytest
    with pytest.raises(fb.FcfdError) as e:
        fb.Case(str(tmp_path / "missing.in"))
    assert e.value.code == 1


def test_unsupported_flux_is_reported(fb, tmp_path):
    import pytest
    from freecfd_b200 import cases
    c = cases.wedge_case(ni=4, nj=3, flux="HLLC")
    with pytest.raises(fb.FcfdError) as e:
        fb.Case(c.write_deck(str(tmp_path)))
    assert e.value.code == 7
