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


SOD_SRC = os.path.join(PKG, "examples", "sod_driver.cpp")


def build_sod_driver(tmp_path):
    exe = str(tmp_path / "sod_driver")
    subprocess.run(["g++", "-std=c++17", "-O2", "-I", os.path.join(ROOT, "include"), SOD_SRC, "-o", exe,
                    "-L", PKG, "-lawcm_b200", f"-Wl,-rpath,{PKG}"], check=True)
    return exe


def test_sod_driver_compiles(tmp_path, awcm_lib):
    assert os.path.exists(build_sod_driver(tmp_path))


@pytest.mark.gpu
def test_sod_driver_matches_oracle(tmp_path, awcm_lib):
    """The 1D mirror (AWCM_1D, AWCM_MANAGER_1D, the facade's wavelet calls) in a compiled driver:
    PrepareEuler pass by pass equals the one-call form, and the Sod run to t = 0.2 equals the
    oracle's (897 steps)."""
    from oracle import Oracle1D

    exe = build_sod_driver(tmp_path)
    out = subprocess.run([exe, "7", "17", "0.2", "1e-4", "0.5", "passes"], capture_output=True, text=True,
                         check=True).stdout.split("\n")
    assert out[0] == "passes equal 1", out[0]
    f = out[1].split()
    steps, t, upd, rho_sum = int(f[1]), float(f[3]), float(f[7]), float(f[9])
    n = 1025
    ref = Oracle1D(7, 17, 0.5 / n, 1 - 0.5 / n, kind="port")
    ref.init_riemann(0.5, (1.0, 0.0, 1.0), (0.125, 0.0, 0.1))
    n_r, t_r, u_r = ref.run(1e-4, 0.5, 0.2)
    assert (steps, t, upd) == (n_r, t_r, u_r) == (897, 0.2, 151533.0)
    acc = 0.0
    for v in ref.get_q()[:, 0]:  # same left-to-right sum as the driver
        acc += float(v)
    assert rho_sum == acc


@pytest.mark.gpu
def test_sod_driver_generic_manager(tmp_path, awcm_lib):
    """The generic BOUNDARY_MANAGER_1D<T> mirror with extrapolation at every ghost cell gives the
    transmissive run."""
    exe = build_sod_driver(tmp_path)
    a = subprocess.run([exe, "7", "17", "0.05", "1e-4", "0.5"], capture_output=True, text=True, check=True).stdout
    b = subprocess.run([exe, "7", "17", "0.05", "1e-4", "0.5", "generic"], capture_output=True, text=True,
                       check=True).stdout
    assert a == b and a.startswith("steps ")
