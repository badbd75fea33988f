"""The enum-driven boundary managers BOUNDARY_MANAGER_1D<T> / BOUNDARY_MANAGER_2D<TT> on the GPU
(awcm1d_batch_set_bc_field, awcm2d_set_bc_field) against the reference's own classes and the CPU
restatement: ghost fills with randomly mixed conditions per ghost cell (corner blocks included),
and steps whose stage fills use the generic manager, bit for bit."""
import numpy as np
import pytest

import oracle
from oracle import Oracle1D, Oracle2D

pytestmark = pytest.mark.gpu


def kinds():
    return ["port", "reference"] if oracle.reference_available() else ["port"]


def random_conditions(shape, seed):
    return np.random.default_rng(seed).integers(-4, 1, size=shape).astype(np.int32)


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_2d_fill_mixed_conditions(awcm_lib, seed):
    geom = (4, 9, 9, 0.0, 1.0, 0.0, 1.0)
    gpu = awcm_lib.AWCM2D(*geom)
    q = np.random.default_rng(seed).uniform(0.5, 2.0, (gpu.ny + 6, gpu.nx + 6, 4))
    bc = random_conditions((gpu.ny + 6, gpu.nx + 6), 100 + seed)
    gpu.set_q(q)
    gpu.set_bc_field(bc)
    gpu.apply_bc()
    for kind in kinds():
        o = Oracle2D(*geom, kind=kind)
        o.set_q(q)
        o.set_bc_field(bc)
        o.apply_bc()
        assert np.array_equal(gpu.get_q(), o.get_q()), kind  # every cell, corners included


def test_2d_steps_with_generic_manager(awcm_lib):
    """Isentropic vortex with periodic conditions in x, extrapolation in y and a SOLID_WALL corner
    block (left as it is): six steps on the GPU and on both checkers."""
    geom = (4, 9, 9, 0.0, 10.0, 0.0, 10.0)
    gpu = awcm_lib.AWCM2D(*geom, bc_kind=2)
    bc = np.full((gpu.ny + 6, gpu.nx + 6), -2, np.int32)
    bc[:, :3] = bc[:, -3:] = -3
    bc[:3, :3] = -4
    gpu.init_problem(2, 5.0, 5.0)
    gpu.set_bc_field(bc)
    refs = []
    for kind in kinds():
        o = Oracle2D(*geom, bc_kind=2, kind=kind)
        o.init_problem(2, 5.0, 5.0)
        o.set_bc_field(bc)
        refs.append(o)
    t = 0.0
    for k in range(6):
        o_g = gpu.step(1e-3, 0.4, t, 10.0)
        for o in refs:
            o_r = o.step(1e-3, 0.4, t, 10.0)
            assert o_g[0] == o_r[0] and np.array_equal(o_g[2:6], o_r[2:6]), (k, o.kind)
        t += o_g[0]
    for o in refs:
        assert np.array_equal(gpu.get_q(), o.get_q()), o.kind
        assert np.array_equal(gpu.get_masks(), o.get_masks()), o.kind
    # the adjoint covers the fixed managers only and says so
    with pytest.raises(awcm_lib.AwcmError, match="generic"):
        gpu.adjoint(t, 1e-3, 2, np.zeros((gpu.ny, gpu.nx)))


def test_1d_fill_and_steps_with_generic_manager(awcm_lib):
    n = 257
    geo = (5, 17, 0.5 / n, 1 - 0.5 / n)
    gpu = awcm_lib.AWCM1D(*geo)
    q = np.random.default_rng(3).uniform(0.5, 2.0, (n + 6, 3))
    for seed in range(4):
        bc = random_conditions(n + 6, 10 + seed)
        gpu.set_q(q)
        gpu.set_bc_field(bc)
        gpu.apply_bc()
        for kind in kinds():
            o = Oracle1D(*geo, kind=kind)
            o.set_q(q)
            o.set_bc_field(bc)
            o.apply_bc()
            assert np.array_equal(gpu.get_q(), o.get_q()), (seed, kind)
    bc = np.full(n + 6, -2, np.int32)
    bc[:3] = -3
    gpu = awcm_lib.AWCM1D(*geo)
    gpu.init_riemann(0.5, (1.0, 0.0, 1.0), (0.125, 0.0, 0.1))
    gpu.set_bc_field(bc)
    refs = []
    for kind in kinds():
        o = Oracle1D(*geo, kind=kind)
        o.init_riemann(0.5, (1.0, 0.0, 1.0), (0.125, 0.0, 0.1))
        o.set_bc_field(bc)
        refs.append(o)
    t = 0.0
    for k in range(20):
        o_g = gpu.step(1e-4, 0.5, t, 0.2)
        for o in refs:
            assert np.array_equal(o_g, o.step(1e-4, 0.5, t, 0.2)), (k, o.kind)
        t += o_g[0]
    for o in refs:
        assert np.array_equal(gpu.get_q(), o.get_q()), o.kind
        assert np.array_equal(gpu.get_masks(), o.get_masks()), o.kind
