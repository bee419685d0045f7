"""The input guards of gtd::system against the reference's own: the units-format check with its
std::invalid_argument message (gregsys.hpp:245-282), the constructor's time-step check
(check_dt, :1401-1405), the setters set_timestep / set_iterations / set_softening /
set_bh_opening_angle (:1636-1672) and check_option (:1406-1411).  The reference side is the
compiled reference headers (oracle/_ref); the tested sides are the Python mirror
(gregpackagescpp_b200.System), the C++ drop-in headers (include/gtd, a program compiled here) and
the C ABI.  Host-only: no GPU is touched."""
import ctypes as C
import math
import os
import subprocess

import numpy as np
import pytest

from gregpackagescpp_b200.system import parse_units

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "gregpackagescpp_b200")

UNITS = [
    "M1:1,D1:1,T1:1", "M66743:66740,D1:1,T1:1", "m1:1,d1:1,t1:1", "  M 1 : 2 , D 3 : 4 , T 5 : 6  ",
    "M01:1,D1:1,T1:1", "M10:1,D1:10,T100:1", "M123456789012345678:1,D1:1,T1:1", "M1:1,D1:1,T1:1\n",
    "M0:1,D1:1,T1:1", "M00:1,D1:1,T1:1", "M1:0,D1:1,T1:1", "M1234567890123456789:1,D1:1,T1:1",
    "M1:1,D1:1", "M1:1;D1:1,T1:1", "X1:1,D1:1,T1:1", "M1:1,D1:1,T1:1,", "M-1:1,D1:1,T1:1", "M1.5:1,D1:1,T1:1",
    "M:1,D1:1,T1:1", "M1:1,D1:1,T1:1 x", "M١:1,D1:1,T1:1", "T1:1,D1:1,M1:1", "M1:1,D1:1,T1:1\t",
]

SETTERS = [  # dt, iterations, eps, theta
    (1.0, 1, 1e-3, 0.5), (0.0, 0, 0.0, math.pi), (-1.0, 2, -1.0, -1e-300), (1e-300, 1, 1e-300, 3.0),
    (float("nan"), 5, float("nan"), float("nan")), (float("inf"), 2 ** 64 - 1, float("inf"), float("inf")),
    (5e-324, 1, 5e-324, 0.0), (1.0, 1, 1.0, math.nextafter(math.pi, 4.0)),
]

OPTIONS = [0, 1, 2, 3, 4, 6, 16, 24, 48, 64, 65536, 16 | 65536, 2 | 65536, 0x30000, 0x20000 | 16, 0x7fffffff,
           -1, -2, 0x10010, 1 << 30, 12345]


@pytest.fixture(scope="module")
def ref():
    from oracle.oracle import RefOracle
    if not RefOracle.available():
        pytest.skip("the reference-backed oracle library was not built here")
    return RefOracle()


@pytest.fixture(scope="module")
def cpp(tmp_path_factory):
    exe = str(tmp_path_factory.mktemp("guards") / "guards")
    cmd = ["g++", "-std=c++20", "-O1", "-I", os.path.join(ROOT, "include"), os.path.join(ROOT, "tests", "cpp", "guards_main.cpp"),
           "-o", exe, "-L", PKG, "-l:libgtd_b200.so", f"-Wl,-rpath,{PKG}"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-4000:]

    def run(lines):
        p = subprocess.run([exe], input="".join(line + "\n" for line in lines), capture_output=True, text=True,
                           timeout=120)
        assert p.returncode == 0, p.stderr
        return p.stdout.splitlines()
    return run


def test_units_python_vs_reference(ref):
    for u in UNITS:
        ok, val = ref.units(u)
        if ok:
            g = parse_units(u)
            assert abs(g - val.value) <= 1e-15 * abs(val.value), (u, g, val.value)
        else:
            with pytest.raises(ValueError) as ei:
                parse_units(u)
            assert str(ei.value) == val, (u, str(ei.value), val)


def test_units_cpp_dropin_vs_reference(ref, cpp):
    lines = [u for u in UNITS if "\n" not in u]
    out = cpp(["units " + u for u in lines])
    for u, got in zip(lines, out):
        ok, val = ref.units(u)
        if ok:
            assert got.startswith("ok "), (u, got)
            assert float.fromhex(got[3:]) == val.value, (u, got)  # same long double arithmetic
        else:
            assert got == "err " + val.replace("\n", "\\n"), (u, got)


def test_empty_units_string_rejected(cpp):
    """The reference's parse_units_format crashes on an empty string (its String operations after
    the failed match fault); both mirrors reject it with the message every other mismatch gets."""
    msg = ('The units_format string passed, "", does not match the format required:\n"Ma:b,Dc:x,Ty:z", where '
           "'a', 'b', 'c', 'x', 'y', and 'z' represent any positive integer number of 1-18 characters starting "
           "with at least one non-zero character.\n")
    with pytest.raises(ValueError) as ei:
        parse_units("")
    assert str(ei.value) == msg
    assert cpp(["units "]) == ["err " + msg.replace("\n", "\\n")]


def test_setters_vs_reference(ref, cpp):
    from gregpackagescpp_b200 import System
    out = cpp([f"set {dt.hex()} {it} {eps.hex()} {th.hex()}" for dt, it, eps, th in SETTERS])
    for (dt, it, eps, th), got in zip(SETTERS, out):
        want = ref.setters(dt, it, eps, th)
        assert tuple(bool(int(b)) for b in got.split()) == want, ((dt, it, eps, th), got, want)
        s = System.__new__(System)  # the setters only touch host fields
        mine = (System.set_timestep(s, dt), System.set_iterations(s, it), System.set_softening(s, eps),
                System.set_bh_opening_angle(s, th))
        assert mine == want, ((dt, it, eps, th), mine, want)


def test_timestep_check_vs_reference(ref, cpp):
    from gregpackagescpp_b200 import System
    values = [1.0, 0.0, -0.0, -3600.0, 5e-324, float("nan"), float("inf")]
    out = cpp([f"dt {d.hex()}" for d in values])
    for d, got in zip(values, out):
        want = ref.construct_dt(d)
        assert got == ("ok" if want is None else "err " + want.replace("\n", "\\n")), (d, got)
        if want is not None:
            with pytest.raises(ValueError) as ei:
                System(np.ones(1), np.zeros((1, 3)), np.zeros((1, 3)), timestep=d)
            assert str(ei.value) == want


def test_check_option_vs_reference(ref):
    from gregpackagescpp_b200 import _lib
    L = _lib.load()
    L.gtd_check_option.argtypes = [C.c_int, C.POINTER(C.c_int)]
    for o in OPTIONS:
        acc = C.c_int(-1)
        _lib.check(L.gtd_check_option(o, C.byref(acc)))
        assert bool(acc.value) == ref.check_option(o), o
