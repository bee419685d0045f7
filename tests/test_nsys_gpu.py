""".nsys snapshots (gregsys.hpp:943-1400 load, 3214-3258 write) against files written by the
reference's own to_nsys and against its loader's verdicts on corrupted copies (tests/golden).

The long doubles in a file (each chunk's restitution coefficient, the header's time and time-step)
are 80-bit values in 16 bytes; their last 6 bytes are padding whose content the reference leaves to
whatever its memory held, so byte comparisons skip them."""
import numpy as np
import pytest

from gregpackagescpp_b200 import NsysFormatError, NsysLoadError, System
from gregpackagescpp_b200.ics import UNITS_G6674, plummer

pytestmark = pytest.mark.gpu

KINDS = {"ddd": ("double", "double", "double"), "fff": ("float", "float", "float"),
         "lll": ("long double", "long double", "long double"), "ffd": ("float", "float", "double")}
CHUNK = {"ddd": 80, "fff": 48, "lll": 144, "ffd": 72}


def _write(tmp_path, name, arr):
    p = tmp_path / f"{name}.nsys"
    p.write_bytes(np.asarray(arr, dtype=np.uint8).tobytes())
    return str(p)


def _not_padding(size, chunk):
    """Byte positions of a file of `size` bytes that are not long-double padding."""
    keep = np.ones(size, bool)
    keep[14:20] = False
    keep[30:36] = False
    for c in range(96, size - chunk + 1, chunk):
        keep[c + 10:c + 16] = False
    return keep


@pytest.mark.parametrize("kind", list(KINDS))
def test_load_reference_files(gpu, golden, tmp_path, kind):
    g = golden
    M, R, T = KINDS[kind]
    s = System.from_nsys(_write(tmp_path, kind, g[f"nsys_{kind}_bytes"]), M=M, R=R, T=T)
    for k, got in (("m", s.m), ("r", s.r), ("rest", s.rest), ("x", s.x), ("v", s.v)):
        assert np.array_equal(got, g[f"nsys_{kind}_{k}"]), k
    t, dt, G = g[f"nsys_{kind}_meta"]
    assert (s.time_elapsed, s.dt, s.G) == (t, dt, G)


@pytest.mark.parametrize("kind", ["ddd", "fff", "ffd"])
def test_write_matches_reference_bytes(gpu, golden, tmp_path, kind):
    """The reference's state after its 3 steps (exact in double for these types) written by this
    engine gives the reference's file."""
    g = golden
    M, R, T = KINDS[kind]
    s = System(g[f"nsys_{kind}_m"], g[f"nsys_{kind}_x"], g[f"nsys_{kind}_v"], r=g[f"nsys_{kind}_r"],
               rest=g[f"nsys_{kind}_rest"], timestep=3600.0, units_format=UNITS_G6674)
    s.time_elapsed = 3 * 3600.0
    p = str(tmp_path / "ours.nsys")
    want = np.asarray(g[f"nsys_{kind}_bytes"], dtype=np.uint8)
    assert s.to_nsys(p, M=M, R=R, T=T) == len(want)
    got = np.frombuffer(open(p, "rb").read(), dtype=np.uint8)
    assert len(got) == len(want) == 96 + 37 * CHUNK[kind]
    keep = _not_padding(len(want), CHUNK[kind])
    assert np.array_equal(got[keep], want[keep])
    assert not got[~keep].any()  # this engine writes zero padding


def test_long_double_roundtrip(gpu, golden, tmp_path):
    """long double M/R/T: the reference's file, re-written here from its (rounded) values, reads
    back to the same values."""
    g = golden
    ld = dict(M="long double", R="long double", T="long double")
    s = System.from_nsys(_write(tmp_path, "lll", g["nsys_lll_bytes"]), **ld)
    p = str(tmp_path / "again.nsys")
    assert s.to_nsys(p, **ld) == 96 + 37 * 144
    t = System.from_nsys(p, **ld)
    for a, b in ((s.m, t.m), (s.r, t.r), (s.rest, t.rest), (s.x, t.x), (s.v, t.v)):
        assert np.array_equal(a, b)


def test_roundtrip_after_mixed_evolve(gpu, tmp_path):
    """The mixed path reorders bodies on the device; the file still holds them in upload order."""
    m, x, v = plummer(3000, 41)
    s = System(m, x, v, timestep=3600.0, num_iterations=20, units_format=UNITS_G6674, precision="mixed")
    s.evolve(System.leapfrog_kdk)
    p = str(tmp_path / "mixed.nsys")
    s.to_nsys(p)
    t = System.from_nsys(p)
    assert np.array_equal(t.x, s.x) and np.array_equal(t.v, s.v) and np.array_equal(t.m, s.m)
    assert t.G == s.G and t.dt == s.dt


def test_corrupted_files_like_reference(gpu, golden, tmp_path):
    g = golden
    for name, rc, msg in zip(g["nsysbad_names"], g["nsysbad_rc"], g["nsysbad_msg"]):
        name, msg = str(name), str(msg)
        path = _write(tmp_path, name, g[f"nsysbad_{name}_bytes"])
        if rc == 0:
            s = System.from_nsys(path)
            t, dt, G, n = g[f"nsysbad_{name}_meta"]
            assert (s.time_elapsed, s.dt, s.G, len(s.m)) == (t, dt, G, n), name
            for k, got in (("m", s.m), ("r", s.r), ("rest", s.rest), ("x", s.x), ("v", s.v)):
                assert np.array_equal(got, g[f"nsysbad_{name}_{k}"]), (name, k)
            continue
        cls = {-1: NsysLoadError, -2: NsysFormatError, -3: ValueError}[int(rc)]
        with pytest.raises(cls) as e:
            System.from_nsys(path)
        if cls is NsysLoadError:
            assert not isinstance(e.value, NsysFormatError), name
        assert str(e.value).endswith(msg), (name, str(e.value), msg)


def test_missing_file_and_null_path(gpu, tmp_path):
    with pytest.raises(NsysLoadError) as e:
        System.from_nsys(str(tmp_path / "absent.nsys"))
    assert str(e.value).endswith("Error obtaining .nsys file information. No data loaded.\n")
    with pytest.raises(NsysLoadError) as e:
        System.from_nsys(str(tmp_path))
    assert str(e.value).endswith(".nsys file provided is not a regular file. Could not load data.\n")
    s = System(*plummer(10, 1))
    assert s.to_nsys(None) == 0
    assert s.to_nsys(str(tmp_path / "no_such_dir" / "f.nsys")) == 0


def test_async_frames_overlap_evolve(gpu, tmp_path):
    """A frame loop with asynchronous snapshots (evolve, to_nsys(wait=False), evolve, ...): every
    file holds the state at its call, bit-identical to a synchronous write of that state."""
    m, x, v = plummer(5000, 71)
    s = System(m, x, v, timestep=3600.0, num_iterations=4, units_format=UNITS_G6674)
    states = []
    for k in range(5):
        s.evolve(System.leapfrog_kdk)
        s.to_nsys(str(tmp_path / f"frame{k}.nsys"), wait=False)
        states.append((s.x.copy(), s.v.copy()))
    assert s.nsys_wait() == 96 + 5000 * 80
    for k, (xk, vk) in enumerate(states):
        t = System.from_nsys(str(tmp_path / f"frame{k}.nsys"))
        assert np.array_equal(t.x, xk) and np.array_equal(t.v, vk)
        ref = System(t.m, xk, vk, units_format=UNITS_G6674)
        p = str(tmp_path / "sync.nsys")
        ref.to_nsys(p)
        a = open(p, "rb").read()
        b = open(str(tmp_path / f"frame{k}.nsys"), "rb").read()
        assert a[96:] == b[96:]
