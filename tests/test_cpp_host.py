"""The C++ host side (include/dem3d_b200.hpp, dem3d_b200/harness/dem_main.cpp):
it compiles against the C-ABI and runs DEM3D's time loop (src/DEM.f90:85-99).
Without a GPU it stops with the no-device status; on a GPU its result is the
oracle's, bit for bit."""
import os
import shutil
import struct
import subprocess

import numpy as np
import pytest

from dem3d_b200 import _abi
from dem3d_b200 import configs

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.join(ROOT, "dem3d_b200")


def build_main(out_dir):
    _abi.load_library()  # builds the library if needed
    exe = os.path.join(out_dir, "dem_main")
    cmd = ["g++", "-std=c++17", "-O2", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"),
           os.path.join(ROOT, "dem3d_b200", "harness", "dem_main.cpp"), "-L", LIBDIR,
           "-l:libdem3d_b200.so", f"-Wl,-rpath,{LIBDIR}", "-o", exe]
    subprocess.run(cmd, check=True)
    return exe


def write_case(path, w, steps, pour=None):
    n = len(w.pos)
    with open(path, "wb") as f:
        f.write(bytes(w.params))
        f.write(struct.pack("<4i", n, steps, pour.interval if pour is not None else 0, 0))
        f.write(np.ascontiguousarray(w.comp, dtype="<i4").tobytes())
        for a in (w.pos, w.vel, w.omega):
            f.write(np.ascontiguousarray(a, dtype="<f8").tobytes())
        if pour is not None:
            f.write(bytes(pour))


def read_out(path):
    data = open(path, "rb").read()
    n = struct.unpack_from("<i", data)[0]
    at = 4
    arrs = []
    for _ in range(3):
        arrs.append(np.frombuffer(data, "<f8", 3 * n, at).reshape(n, 3))
        at += 24 * n
    comp = np.frombuffer(data, "<i4", n, at)
    ncol = struct.unpack_from("<q", data, at + 4 * n)[0]
    return arrs, comp, ncol


@pytest.mark.skipif(shutil.which("g++") is None, reason="no C++ compiler")
def test_cpp_main_builds_and_reports_no_device(tmp_path):
    exe = build_main(str(tmp_path))
    case = os.path.join(tmp_path, "case.bin")
    write_case(case, configs.settling(n=300, seed=2, sigma_v=0.5), 10)
    r = subprocess.run([exe, case, os.path.join(tmp_path, "out.bin")], capture_output=True,
                       text=True)
    if r.returncode == 3:
        assert "no CUDA device" in r.stderr
    else:  # a GPU is present
        assert r.returncode == 0, r.stderr
    bad = subprocess.run([exe, os.path.join(tmp_path, "missing.bin"), "x"], capture_output=True)
    assert bad.returncode == 2


@pytest.mark.gpu
def test_cpp_main_equals_the_oracle(tmp_path):
    from tests.oracle_lib import oracle_system
    exe = build_main(str(tmp_path))
    w = configs.settling(n=300, seed=2, sigma_v=0.5)
    case, out = os.path.join(tmp_path, "case.bin"), os.path.join(tmp_path, "out.bin")
    write_case(case, w, 400)
    r = subprocess.run([exe, case, out], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    (pos, vel, omega), comp, ncol = read_out(out)
    o = oracle_system(w.params)
    o.set_state(w.pos, w.vel, w.omega, comp=w.comp)
    o.initialize_cell_distribution()
    o.run(1, 400)
    st = o.get_state()
    np.testing.assert_array_equal(pos, st["pos"])
    np.testing.assert_array_equal(vel, st["vel"])
    np.testing.assert_array_equal(omega, st["omega"])
    assert ncol == o.ncol() > 0


def _oracle_run(w, steps, pour=None):
    from tests.oracle_lib import oracle_system
    o = oracle_system(w.params)
    o.set_state(w.pos, w.vel, w.omega, comp=w.comp)
    o.initialize_cell_distribution()
    if pour is not None:
        o.set_pouring(pour)
    o.run(1, steps)
    return o


@pytest.mark.gpu
def test_cpp_main_fewer_steps_than_the_start_up(tmp_path):
    """NumberOfSteps = 1 < MethodOrder - 1: the start-up still runs its
    MethodOrder - 1 Euler steps (src/DEM.f90:88-90), as the oracle does."""
    exe = build_main(str(tmp_path))
    w = configs.settling(n=300, seed=2, sigma_v=0.5)
    case, out = os.path.join(tmp_path, "case.bin"), os.path.join(tmp_path, "out.bin")
    write_case(case, w, 1)
    r = subprocess.run([exe, case, out], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    (pos, vel, omega), comp, ncol = read_out(out)
    st = _oracle_run(w, 1).get_state()
    np.testing.assert_array_equal(pos, st["pos"])
    np.testing.assert_array_equal(vel, st["vel"])
    assert not np.array_equal(pos, w.pos)


@pytest.mark.gpu
def test_cpp_main_pouring_equals_the_oracle(tmp_path):
    """PouringAttempt before MoveParticles every IPouring steps, through the
    C++ time loop: the same spheres go in at the same places."""
    from types import SimpleNamespace
    from tests.test_pouring import filling_box
    exe = build_main(str(tmp_path))
    prm, pos, comp, pour = filling_box(interval=4)
    w = SimpleNamespace(params=prm, pos=pos, vel=np.zeros_like(pos), omega=np.zeros_like(pos),
                        comp=comp)
    case, out = os.path.join(tmp_path, "case.bin"), os.path.join(tmp_path, "out.bin")
    write_case(case, w, 400, pour=pour)
    r = subprocess.run([exe, case, out], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    (gpos, gvel, gomega), gcomp, ncol = read_out(out)
    o = _oracle_run(w, 400, pour)
    st = o.get_state()
    assert len(gpos) == o.n > len(pos)
    np.testing.assert_array_equal(gpos, st["pos"])
    np.testing.assert_array_equal(gvel, st["vel"])
    np.testing.assert_array_equal(gomega, st["omega"])
    np.testing.assert_array_equal(gcomp, o.comp)
    assert ncol == o.ncol()
