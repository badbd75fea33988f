"""The C++ mirror classes (include/awcm_b200.hpp) compile against the C-ABI, and a driver written
like the reference's main loop gives the same run as the oracle."""
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "c_pp-library_b200")
SRC = os.path.join(PKG, "examples", "quadrants_driver.cpp")


def build_driver(tmp_path, awcm):
    exe = str(tmp_path / "quadrants_driver")
    subprocess.run(["g++", "-std=c++17", "-O2", "-I", os.path.join(ROOT, "include"), SRC, "-o", exe,
                    "-L", PKG, "-lawcm_b200", f"-Wl,-rpath,{PKG}"], check=True)
    return exe


def test_driver_compiles(tmp_path, awcm_lib):
    assert os.path.exists(build_driver(tmp_path, awcm_lib))


@pytest.mark.gpu
def test_driver_matches_oracle(tmp_path, awcm_lib):
    from oracle import Oracle2D

    exe = build_driver(tmp_path, awcm_lib)
    out = subprocess.run([exe, "4", "9", "0.02", "1e-3", "0.4"], capture_output=True, text=True, check=True).stdout
    f = out.split()
    steps, t, upd, rho_sum = int(f[1]), float(f[3]), float(f[7]), float(f[9])
    ref = Oracle2D(4, 9, 9, 0.0, 1.0, 0.0, 1.0, kind="port")
    ref.init_problem(0, 0.5, 0.5)
    n, t_r, u_r = ref.run(1e-3, 0.4, 0.02)
    assert (steps, t, upd) == (n, t_r, u_r)
    acc = 0.0
    for v in ref.get_q().reshape(-1, 4)[:, 0]:  # same left-to-right sum as the driver
        acc += float(v)
    assert rho_sum == acc
