"""The C ABI library loads and exports every entry point include/gtd_b200.h declares (no compute
calls: this runs on machines without a GPU)."""
import ctypes as C
import os
import subprocess

from gregpackagescpp_b200 import _lib


def test_library_exports_every_declared_symbol():
    L = _lib.load()
    declared = _lib.exported_symbols()
    assert len(declared) >= 20
    for name in declared:
        assert hasattr(L, name), name
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.LIB_PATH], capture_output=True, text=True).stdout
    exported = {ln.split()[-1] for ln in out.splitlines() if " T " in ln}
    assert set(declared) <= exported
    # nothing else leaks out of the library
    assert {s for s in exported if not s.startswith("gtd_")} == set()


def test_abi_version_and_error_channel():
    L = _lib.load()
    assert L.gtd_abi_version() == 1
    # a NULL handle is rejected with a message, without touching a device
    assert L.gtd_system_set_params(None, 1.0, 1.0, 1, 0.0, 0.5) == _lib.ERR_INVALID_ARGUMENT
    assert b"NULL" in L.gtd_last_error()
    assert L.gtd_system_destroy(None) == 0


def test_header_compiles_as_c_and_cxx(tmp_path):
    inc = os.path.join(os.path.dirname(_lib.PKG), "include")
    src = tmp_path / "t.c"
    src.write_text('#include "gtd_b200.h"\nint main(void){return gtd_abi_version()==GTD_ABI_VERSION?0:1;}\n')
    for cc, extra in (("gcc", ["-std=c99"]), ("g++", ["-x", "c++", "-std=c++20"])):
        r = subprocess.run([cc, *extra, "-I", inc, "-c", str(src), "-o", str(tmp_path / "t.o")],
                           capture_output=True, text=True)
        assert r.returncode == 0, r.stderr
