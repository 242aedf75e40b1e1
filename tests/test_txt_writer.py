"""The text output of the drop-in (writeFinalResultTo_txt) against the
reference's own writer, byte for byte, without a GPU.

The reference writes rho_/p_/u_/v_<t>s.txt with its protected static
writeMatrixTo_txt (src/wrappers.cuh:370-397, reached from
writeFinalResultTo_txt at src/wrappers.cuh:318-321).  oracle/_ref/ref_txt is
that function compiled unchanged from the reference's header (oracle/ref_txt.cu,
built by oracle/Makefile where the reference sources are present).  Both
mirrors -- the C++ header's writeFinalResultTo_txt (include/rgrp_2d_cuda.hpp)
and the Python class's (2d_fvm_cuda_b200/solver.py, write_matrix_txt) --
must produce the same four files, names included."""
import os
import struct
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_TXT = os.path.join(ROOT, "oracle", "_ref", "ref_txt")
LIBDIR = os.path.join(ROOT, "2d_fvm_cuda_b200", "lib")


def state(seed):
    """Values the default stream format treats differently: integers, signs,
    signed zero, six-digit rounding, exponent forms, infinities."""
    r = np.random.default_rng(seed)
    ny, nx = 7, 9
    U = r.normal(size=(ny, nx, 4)) * 10.0 ** r.integers(-9, 9, size=(ny, nx, 4))
    U[0, :4, 0] = [1.0, -0.0, 0.0, 123456.5]
    U[1, :5, 1] = [1e-5, 1e-4, 999999.5, 1234567.0, -2.5e-300]
    U[2, :3, 2] = [np.inf, -np.inf, 100000.0]
    U[3, :3, 3] = [0.1 + 0.2, 2.0 / 3.0, -1e16]
    return U


def write_input(path, U, t):
    ny, nx = U.shape[:2]
    with open(path, "wb") as f:
        f.write(struct.pack("<iid", nx, ny, t))
        f.write(np.ascontiguousarray(U[..., :4], dtype="<f8").tobytes())


def files(d):
    return {n: open(os.path.join(d, n), "rb").read() for n in sorted(os.listdir(d))}


@pytest.mark.skipif(not os.path.exists(REF_TXT), reason="reference text writer not built (reference sources absent)")
@pytest.mark.parametrize("t", [0.2, 0.35, 1.0 / 3.0, 10.0])
def test_text_files_equal_the_reference_writer(pkg, tmp_path, t):
    U = state(int(t * 1000))
    inp = str(tmp_path / "state.bin")
    write_input(inp, U, t)
    ref_dir, py_dir, cpp_dir = (tmp_path / d for d in ("ref", "py", "cpp"))
    for d in (ref_dir, py_dir, cpp_dir):
        d.mkdir()
    subprocess.run([REF_TXT, inp, str(ref_dir)], check=True)
    pkg.solver.write_matrix_txt(str(py_dir), U, t)
    exe = str(tmp_path / "txt_driver")
    subprocess.run(["g++", "-std=c++17", "-O2", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "txt_driver.cpp"), "-L", LIBDIR, "-lfvm2d",
                    f"-Wl,-rpath,{LIBDIR}", "-o", exe], check=True)
    subprocess.run([exe, inp, str(cpp_dir)], check=True)
    R = files(ref_dir)
    assert sorted(R) == [f"{n}_{'%f' % t}s.txt" for n in ("p", "rho", "u", "v")]
    assert files(py_dir) == R
    assert files(cpp_dir) == R
