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


def test_struct_layouts_match_header(fb, tmp_path):
    """The ctypes mirrors of the option and report structs have the header's
    layout: a C program compiled against include/fcfd.h prints each struct's
    size and every member's offset (members named as in the mirror)."""
    import shutil
    import subprocess
    import pytest
    from freecfd_b200 import _lib
    if shutil.which("gcc") is None:
        pytest.skip("no C compiler")
    mirrors = {"fcfd_newton_opts": _lib.NewtonOpts, "fcfd_newton_report": _lib.NewtonReport,
               "fcfd_run_opts": _lib.RunOpts, "fcfd_run_report": _lib.RunReport, "fcfd_raw_mesh": _lib._RawMesh}
    lines = ["#include <stddef.h>", "#include <stdio.h>", '#include "fcfd.h"', "int main(void) {"]
    for cname, cls in mirrors.items():
        lines.append(f'  printf("{cname} size %zu\\n", sizeof({cname}));')
        for f in cls._fields_:
            lines.append(f'  printf("{cname} {f[0]} %zu\\n", offsetof({cname}, {f[0]}));')
    lines += ["  return 0;", "}"]
    src, exe = tmp_path / "layout.c", tmp_path / "layout"
    src.write_text("\n".join(lines) + "\n")
    subprocess.run(["gcc", "-std=c11", "-I", os.path.join(ROOT, "include"), "-o", str(exe), str(src)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n")
    got = {tuple(ln.split()[:2]): int(ln.split()[2]) for ln in out if ln}
    for cname, cls in mirrors.items():
        assert got[(cname, "size")] == ctypes.sizeof(cls), cname
        for f in cls._fields_:
            assert got[(cname, f[0])] == getattr(cls, f[0]).offset, (cname, f[0])
