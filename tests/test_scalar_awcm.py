"""Scalar AWCM path (Wavelet/main_2d_advect.cpp): the CPU restatement against the reference's own
code, and the CUDA path against the restatement, bit for bit.  Workload: the driver's Gaussian
exp(-50 (x-0.5)^2 - 50 (y-0.5)^2) (Problems/2D/PROBLEM_BOX_ADVECTION.h:45-52) on cell-centred
nodes of [0,1]^2, periodic, dt = 0.4 dx, threshold 1e-4."""
import numpy as np
import pytest

import oracle
from oracle import Oracle2D


def geometry(num_levels, nx_coarse):
    n = (nx_coarse - 1) * 2 ** (num_levels - 1) + 1
    d = 1.0 / n
    return (num_levels, nx_coarse, nx_coarse, 0.5 * d, 1 - 0.5 * d, 0.5 * d, 1 - 0.5 * d), n, d


def gaussian(n, d):
    x = 0.5 * d + (np.arange(n + 6) - 3) * d
    X, Y = np.meshgrid(x, x)
    return np.exp(-50 * (X - 0.5) ** 2 - 50 * (Y - 0.5) ** 2)


def checker(kind, geom):
    o = Oracle2D(*geom, bc_kind=2, kind=kind)
    o.set_scalar()
    return o


@pytest.mark.parametrize("levels,nxc,steps", [(4, 9, 12), (5, 15, 6)])
def test_restatement_matches_reference(levels, nxc, steps):
    if not oracle.reference_available():
        pytest.skip("reference build absent")
    geom, n, d = geometry(levels, nxc)
    q0 = gaussian(n, d)
    a, b = checker("port", geom), checker("reference", geom)
    for o in (a, b):
        o.scalar_set_q(q0)
    for k in range(steps):
        oa, ob = a.scalar_step(1e-4, 0.4 * d), b.scalar_step(1e-4, 0.4 * d)
        assert np.array_equal(oa, ob), k
        assert np.array_equal(a.scalar_get_q()[3:-3, 3:-3], b.scalar_get_q()[3:-3, 3:-3]), k
        assert np.array_equal(a.get_masks(), b.get_masks()), k
        assert np.array_equal(a.get_levels()[:3], b.get_levels()[:3]), k


def test_advection_moves_the_blob():
    """After 60 steps at unit velocity the density maximum has moved by about 60 * 0.4 dx in
    both directions and the field stays within its initial range."""
    geom, n, d = geometry(4, 9)
    a = checker("port", geom)
    q0 = gaussian(n, d)
    a.scalar_set_q(q0)
    for _ in range(60):
        a.scalar_step(1e-4, 0.4 * d)
    q = a.scalar_get_q()[3:-3, 3:-3]
    j, i = np.unravel_index(np.argmax(q), q.shape)
    shift = 60 * 0.4 * d
    assert abs((i * d + 0.5 * d) - (0.5 + shift)) < 2 * d and abs((j * d + 0.5 * d) - (0.5 + shift)) < 2 * d
    assert q.max() <= 1.0 + 1e-6 and q.min() >= -1e-3


@pytest.mark.gpu
@pytest.mark.parametrize("levels,nxc,steps", [(4, 9, 12), (6, 15, 20)])
def test_gpu_matches_restatement(levels, nxc, steps, awcm_lib):
    import ctypes

    geom, n, d = geometry(levels, nxc)
    q0 = gaussian(n, d)
    o = checker("port", geom)
    o.scalar_set_q(q0)
    s = awcm_lib.AWCM2DScalar(*geom)
    s.set_q(q0)
    t, dt = 0.0, 0.4 * d
    for k in range(steps):
        out = o.scalar_step(1e-4, dt)
        t2, m, upd = s.advance(1e-4, dt, t, 1)
        assert m == 1 and upd == out[0], (k, upd, out)
        t = t2
        assert np.array_equal(s.get_q()[3:-3, 3:-3], o.scalar_get_q()[3:-3, 3:-3]), k
    assert np.array_equal(s.get_masks(), o.get_masks())
    assert np.array_equal(s.get_levels()[:3], o.get_levels()[:3])


@pytest.mark.gpu
def test_gpu_scalar_rejects_euler_calls(awcm_lib):
    geom, n, d = geometry(4, 9)
    s = awcm_lib.AWCM2DScalar(*geom)
    with pytest.raises(awcm_lib.AwcmError, match="ERR_STATE"):
        awcm_lib._lib.call("awcm2d_step", s.h, 1e-4, 0.4, 0.0, 1.0, 0.0, None)
