"""Code written against the reference's C++ API (gtd::system, gtd::body, gtd::bh_tree) compiles
unchanged against include/gtd/*.hpp and links the C ABI library; on a GPU it runs and agrees with
the CPU oracle (tests/cpp/dropin_main.cpp)."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cpp", "dropin_main.cpp")
PKG = os.path.join(ROOT, "gregpackagescpp_b200")
ORC = os.path.join(ROOT, "oracle")


def build(out):
    from oracle.oracle import ensure_built
    ensure_built()
    cmd = ["g++", "-std=c++20", "-O2", "-I", os.path.join(ROOT, "include"), "-I", ORC, SRC, "-o", out,
           "-L", PKG, "-l:libgtd_b200.so", "-L", ORC, "-l:liboracle.so", f"-Wl,-rpath,{PKG}", f"-Wl,-rpath,{ORC}"]
    return subprocess.run(cmd, capture_output=True, text=True)


def test_dropin_headers_compile_and_link(tmp_path):
    r = build(str(tmp_path / "dropin"))
    assert r.returncode == 0, r.stderr[-4000:]


@pytest.mark.gpu
def test_dropin_program_runs_on_gpu(gpu, tmp_path):
    exe = str(tmp_path / "dropin")
    r = build(exe)
    assert r.returncode == 0, r.stderr[-4000:]
    run = subprocess.run([exe], capture_output=True, text=True, timeout=600)
    print(run.stdout)
    assert run.returncode == 0, run.stdout + run.stderr
