"""The C++ drop-in: tests/drop_in_driver.cpp is written against the
reference's RGRP_2D_CUDA class; it must build with a plain host compiler
against include/rgrp_2d_cuda.hpp and libfvm2d.so, and on the GPU give what
the Python mirror of the same class gives (same library, same build: bit for
bit), frames included."""
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.join(ROOT, "2d_fvm_cuda_b200", "lib")


def build(tmp_path):
    exe = str(tmp_path / "drop_in_driver")
    subprocess.run(["g++", "-std=c++17", "-O2", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "drop_in_driver.cpp"), "-L", LIBDIR, "-lfvm2d",
                    f"-Wl,-rpath,{LIBDIR}", "-o", exe], check=True)
    return exe


def test_reference_program_builds_against_the_header(pkg, tmp_path):
    assert os.path.exists(build(tmp_path))


@pytest.mark.gpu
@pytest.mark.parametrize("strategy", [0, 4])
def test_reference_program_matches_the_python_mirror(pkg, tmp_path, strategy):
    exe = build(tmp_path)
    out, frames = str(tmp_path / "out.bin"), str(tmp_path / "frames")
    subprocess.run([exe, "64", str(strategy), out, frames], check=True)
    raw = open(out, "rb").read()
    n, steps = np.frombuffer(raw[:8], np.int32)
    U = np.frombuffer(raw[16:], np.float64).reshape(n, n, 5)
    s = pkg.RGRP_2D_CUDA()
    s.setRPInitialData([1.5, 1.5, 0.0, 0.0], [0.5323, 0.3, 1.206, 0.0], [0.138, 0.029, 1.206, 1.206],
                       [0.5323, 0.3, 0.0, 1.206], 64, 64)
    s.setSpatialLayout(1.0, 1.0)
    s.setTimeLayout(0.05, 0.45)
    s.setAlpha(1.9)
    s.setGamma(1.4)
    s.setGhostCellStrategy(strategy)
    V = s.solve()
    assert steps == s.getTimeStagesCount()
    assert np.array_equal(U[..., :4], V[..., :4])
    assert sorted(os.listdir(frames), key=lambda x: int(x.split(".")[0])) == [f"{k}.png" for k in range(0, steps, 10)]
