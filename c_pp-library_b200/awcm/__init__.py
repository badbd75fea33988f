"""awcm -- B200-native AWCM compressible-Euler path (host side).

The compute runs in libawcm_b200.so (hand-written CUDA for sm_100a behind the C-ABI of
include/awcm_b200.h); this package binds it with ctypes and mirrors the reference's call surface.
"""
from ._lib import AwcmError, LIB_PATH, exported_symbols, load
from .solvers import (EXTRAPOLATION_ZERO_ORDER, FLUID, PERIODIC, SOLID_WALL, SPECIFIED, BC_GENERIC, BC_SHOCK_VORTEX,
                      BC_WIND_TUNNEL, PROBLEM_SHOCK_VORTEX, PROBLEM_WIND_TUNNEL, AAZ, APD, BAND, BC_DOUBLE_MACH, BC_PERIODIC, BC_TRANSMISSIVE, CL, CR, PROBLEM_DOUBLE_MACH,
                      PROBLEM_QUADRANTS, PROBLEM_VORTEX, RR, SCALAR_ADVECTION, WENO5, WENOZ, AWCM1D, AWCM1DBatch, AWCM1DScalar, AWCM2D,
                      AWCM2DScalar, euler_flux, euler_spectral_radius,
                      measure_fp64_peak)

__all__ = [
    "AwcmError", "measure_fp64_peak", "euler_flux", "euler_spectral_radius", "LIB_PATH", "exported_symbols", "load", "AWCM1D", "AWCM1DBatch", "AWCM1DScalar", "AWCM2D", "AWCM2DScalar",
    "AAZ", "CR", "APD", "CL", "RR", "BAND", "BC_TRANSMISSIVE", "BC_DOUBLE_MACH", "BC_PERIODIC",
    "PROBLEM_QUADRANTS", "PROBLEM_DOUBLE_MACH", "PROBLEM_VORTEX", "WENOZ", "WENO5", "SCALAR_ADVECTION",
    "SOLID_WALL", "PERIODIC", "EXTRAPOLATION_ZERO_ORDER", "SPECIFIED", "FLUID", "BC_GENERIC", "BC_SHOCK_VORTEX",
    "BC_WIND_TUNNEL", "PROBLEM_SHOCK_VORTEX", "PROBLEM_WIND_TUNNEL",
]
