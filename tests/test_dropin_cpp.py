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


def _ref_driver():
    from oracle.oracle import reference_tree
    tree = reference_tree()
    return os.path.join(tree, "nrg.cpp") if tree else None


REF_DRIVER = _ref_driver()


@pytest.mark.skipif(REF_DRIVER is None or not os.path.exists(REF_DRIVER), reason="the reference tree is not here")
def test_reference_driver_compiles_unchanged(tmp_path):
    """nrg.cpp, one of the reference's own drivers (it loads .nsys files into
    gtd::system<T,T,T,true,false,3,0,0,false> for three T and sums their energies through body and
    vector3D accessors), compiles unchanged against include/gtd and links the engine.  The source is
    copied to a scratch directory first, so that its own directory's headers do not shadow these."""
    import shutil
    src = tmp_path / "nrg.cpp"
    shutil.copy(REF_DRIVER, src)
    cmd = ["g++", "-std=c++20", "-O1", "-I", os.path.join(ROOT, "include", "gtd"), "-I", os.path.join(ROOT, "include"),
           str(src), "-o", str(tmp_path / "nrg"), "-L", PKG, "-l:libgtd_b200.so", f"-Wl,-rpath,{PKG}"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-4000:]


@pytest.mark.gpu
def test_tree_walk_program_matches_reference(gpu, tmp_path):
    """tests/cpp/tree_walk_main.cpp is written against the reference's bh_tree API only (begin/end
    over leaves, cell_begin with its cell_iterator, nn_begin, cube_mass, cube_com, operator[]).
    Compiled against the drop-in headers it builds the octree on the GPU and walks the downloaded
    cells; its output equals the same program's output against the reference headers
    (tests/golden/tree_walk_ref.txt, made by tests/golden/make_golden.py): the leaf order, every
    body's cell and neighbour counts and the children listed exactly, the force sums within 1e-12."""
    import numpy as np
    exe = str(tmp_path / "tree_walk")
    cmd = ["g++", "-std=c++20", "-O2", "-I", os.path.join(ROOT, "include", "gtd"), "-I", os.path.join(ROOT, "include"),
           os.path.join(ROOT, "tests", "cpp", "tree_walk_main.cpp"), "-o", exe, "-L", PKG, "-l:libgtd_b200.so",
           f"-Wl,-rpath,{PKG}"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-4000:]
    run = subprocess.run([exe, "2000"], capture_output=True, text=True, timeout=600)
    assert run.returncode == 0, run.stderr
    got = run.stdout.splitlines()
    want = open(os.path.join(ROOT, "tests", "golden", "tree_walk_ref.txt")).read().splitlines()
    assert len(got) == len(want)
    worst = 0.0
    for g, w in zip(got, want):
        if not g[0].isdigit():  # the children lines and the opening-angle line
            assert g == w
            continue
        gi, wi = g.split(), w.split()
        assert gi[:3] == wi[:3], (g, w)  # body index (leaf order), cell count, neighbour count
        ga, wa = np.array([float(t) for t in gi[3:]]), np.array([float(t) for t in wi[3:]])
        worst = max(worst, float(np.abs(ga - wa).max() / np.abs(wa).max()))
    assert worst < 1e-12, worst
