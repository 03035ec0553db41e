"""The C ABI without a GPU: the library loads, exports every entry point declared in
include/nadvibs.h, host-only handles work, device calls fail loudly, and a C driver compiles
against the header and links against the library."""
import os
import re
import subprocess

import pytest

from nadvibs_b200 import _lib as L
from nadvibs_b200 import synth

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    text = open(os.path.join(ROOT, "include", "nadvibs.h")).read()
    return re.findall(r"^(?:int|const char \*)\s*(nvb_\w+)\(", text, re.M)


def test_library_exports_every_declared_symbol():
    lib = L.lib()
    names = _declared()
    assert len(names) >= 25
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    out = subprocess.run(["nm", "-D", "--defined-only", L.LIB_PATH], capture_output=True, text=True).stdout
    for n in names:
        assert re.search(rf"\bT {n}\b", out), n


def test_host_only_handle_and_loud_device_errors(tmp_path):
    b, n = synth.write_inputs(str(tmp_path), synth.config(1))
    with L.Handle.from_files(b, n, device=-1) as h:
        assert h.sizes()["dimen"] == 2304 and len(h.terms()) == 14
        h.write_header(str(tmp_path / "output.dat"))
        assert "Dimensionality of a single State Vector:            2304" in (tmp_path / "output.dat").read_text()
        for call in (lambda: h.seed(), lambda: h.lanczos(2), lambda: h.hv_ptr(1, 2, 0)):
            with pytest.raises(L.NvbError) as e:
                call()
            assert e.value.code in (-3, -4)


def test_c_driver_compiles_and_links(tmp_path):
    exe = tmp_path / "nadvibs_driver"
    r = subprocess.run(["gcc", "-O2", "-I", os.path.join(ROOT, "include"),
                        os.path.join(ROOT, "nadvibs_b200", "examples", "nadvibs_driver.c"), "-o", str(exe),
                        "-L", os.path.join(ROOT, "nadvibs_b200"), "-lnadvibs_gpu",
                        f"-Wl,-rpath,{os.path.join(ROOT, 'nadvibs_b200')}"], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


def test_fortran_interface_names_exist():
    """Every bind(C, name=...) of the Fortran module names an exported entry point."""
    text = open(os.path.join(ROOT, "nadvibs_b200", "fortran", "nadvibs_gpu.f90")).read()
    names = re.findall(r'bind\(C, name="(nvb_\w+)"\)', text)
    assert len(names) >= 10
    lib = L.lib()
    assert all(hasattr(lib, n) for n in names)
