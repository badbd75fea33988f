"""The CPU restatement against the reference itself (compiled from the reference tree), on cases
beyond the committed fixtures.  Skipped where the reference build is absent."""
import numpy as np
import pytest

import oracle
from oracle import Oracle1D, Oracle2D

pytestmark = pytest.mark.skipif(not oracle.reference_available(), reason="reference build (oracle/_ref) absent")


def corner_free(q):
    keep = np.ones(q.shape[:2], bool)
    keep[:3, :3] = keep[:3, -3:] = keep[-3:, :3] = keep[-3:, -3:] = False
    return q[keep]


@pytest.mark.parametrize("scheme", [0, 1])
def test_1d_sod_long(scheme):
    n = 1025
    a = Oracle1D(7, 17, 0.5 / n, 1 - 0.5 / n, scheme=scheme, kind="port")
    b = Oracle1D(7, 17, 0.5 / n, 1 - 0.5 / n, scheme=scheme, kind="reference")
    for o in (a, b):
        o.init_riemann(0.5, (1.0, 0.0, 1.0), (0.125, 0.0, 0.1))
    t = 0.0
    for k in range(300):
        oa, ob = a.step(1e-4, 0.5, t, 0.2), b.step(1e-4, 0.5, t, 0.2)
        assert np.array_equal(oa, ob), k
        t += oa[0]
    assert np.array_equal(a.get_q(), b.get_q())
    assert np.array_equal(a.get_masks(), b.get_masks())
    assert np.array_equal(a.get_levels(), b.get_levels())


def test_1d_shipped_driver_geometry():
    """The shipped driver's own grid: 16 coarse points, 11 levels, [0,10], tol 1e-6 (first steps)."""
    nx = 15 * 2 ** 10 + 1
    dxf = 10.0 / nx
    a = Oracle1D(11, 16, 0.5 * dxf, 10 - 0.5 * dxf, scheme=1, kind="port")
    b = Oracle1D(11, 16, 0.5 * dxf, 10 - 0.5 * dxf, scheme=1, kind="reference")
    for o in (a, b):
        o.init_riemann(5.0, (1.0, 0.0, 1.0), (0.125, 0.0, 0.1))
    t = 0.0
    for k in range(20):
        oa, ob = a.step(1e-6, 0.5, t, 2.0), b.step(1e-6, 0.5, t, 2.0)
        assert np.array_equal(oa, ob), k
        t += oa[0]
    assert np.array_equal(a.get_q(), b.get_q())


@pytest.mark.parametrize("case", [
    (6, 17, 17, (0.0, 1.0, 0.0, 1.0), 0, 0, 0.5, 0.5, 1e-3, 0.4, 2),   # 513^2 quadrants
    (5, 17, 5, (0.0, 4.0, 0.0, 1.0), 1, 1, 1.5, 0.0, 1e-3, 0.5, 3),   # double Mach, reference IC density 1.5
    (5, 9, 9, (0.0, 10.0, -5.0, 5.0), 2, 2, 5.0, 0.0, 1e-3, 0.4, 3),  # vortex at the reference's centre
    (5, 9, 9, (-16.0, 8.0, -12.0, 12.0), 3, 3, 2.0, 0.0, 1e-3, 0.4, 4),  # shock-vortex, reference domain
])
def test_2d_cases(case):
    nl, nxc, nyc, dom, bc, prob, a_, b_, tol, cfl, steps = case
    a = Oracle2D(nl, nxc, nyc, *dom, bc_kind=bc, kind="port")
    b = Oracle2D(nl, nxc, nyc, *dom, bc_kind=bc, kind="reference")
    for o in (a, b):
        o.init_problem(prob, a_, b_)
    assert np.array_equal(a.get_q(), b.get_q())
    t = 0.0
    for k in range(steps):
        oa, ob = a.step(tol, cfl, t, 10.0), b.step(tol, cfl, t, 10.0)
        assert np.array_equal(oa, ob), k
        t += oa[0]
        assert np.array_equal(corner_free(a.get_q()), corner_free(b.get_q()))
        assert np.array_equal(a.get_masks(), b.get_masks())
        assert np.array_equal(a.get_levels()[:3], b.get_levels()[:3])


def test_2d_passes_individually():
    a = Oracle2D(5, 9, 9, 0.0, 1.0, 0.0, 1.0, kind="port")
    b = Oracle2D(5, 9, 9, 0.0, 1.0, 0.0, 1.0, kind="reference")
    for o in (a, b):
        o.init_problem(0, 0.5, 0.5)
        o.fwt(1e-3)
    assert np.array_equal(a.get_q(), b.get_q()) and np.array_equal(a.get_masks(), b.get_masks())
    for op, mask_id, level_id in [(oracle.BAND, 0, 0), (oracle.AAZ, 0, 0), (oracle.CR, 0, 0), (oracle.CL, 0, 0),
                                  (oracle.APD, 0, 0), (oracle.CR, 0, 0), (oracle.RR, 0, 0)]:
        a.manager(op, mask_id, level_id)
        b.manager(op, mask_id, level_id)
        assert np.array_equal(a.get_masks(), b.get_masks()), op
        assert np.array_equal(a.get_levels()[0], b.get_levels()[0]), op
        assert np.array_equal(a.get_q(), b.get_q()), op
    for o in (a, b):
        o.iwt(0)
        o.interpolate(4, 0)
    assert np.array_equal(a.get_q(), b.get_q())


@pytest.mark.parametrize("dim,direction", [(1, 0), (2, 0), (2, 1)])
def test_euler_equation_batch(dim, direction):
    """EULER_EQUATION_1D/2D: the restatement's fluxes and spectral radii equal the reference class's."""
    rng = np.random.default_rng(5 + dim + direction)
    n = 4096
    rho = 10.0 ** rng.uniform(-2, 2, n)
    p = 10.0 ** rng.uniform(-2, 2, n)
    vel = rng.uniform(-3, 3, (n, dim))
    q = np.column_stack([rho, rho[:, None] * vel, p / 0.4 + 0.5 * rho * (vel ** 2).sum(axis=1)])
    assert np.array_equal(oracle.euler_flux(q, dim, direction, kind="port"),
                          oracle.euler_flux(q, dim, direction, kind="reference"))
    assert np.array_equal(oracle.euler_spectral_radius(q, dim, direction, kind="port"),
                          oracle.euler_spectral_radius(q, dim, direction, kind="reference"))


def test_1d_interpolate_and_boundary_fill():
    """WAVELET_1D::InterpolateEuler(mask_temp -> mask3) on a stepped state with a perturbed field,
    and the transmissive ghost fill: restatement equal to the reference."""
    n = 1025
    a = Oracle1D(7, 17, 0.5 / n, 1 - 0.5 / n, kind="port")
    b = Oracle1D(7, 17, 0.5 / n, 1 - 0.5 / n, kind="reference")
    for o in (a, b):
        o.init_riemann(0.5, (1.0, 0.0, 1.0), (0.125, 0.0, 0.1))
    t = 0.0
    for _ in range(40):
        t += a.step(1e-4, 0.5, t, 0.2)[0]
        b.step(1e-4, 0.5, t, 0.2)
    q = a.get_q() + np.random.default_rng(3).uniform(0, 1e-3, a.get_q().shape)
    for o in (a, b):
        o.set_q(q)
        o.interpolate(4, 3)
    assert np.array_equal(a.get_q(), b.get_q())
    for o in (a, b):
        o.apply_bc()
    assert np.array_equal(a.get_q(), b.get_q())


def random_conditions(shape, seed):
    """A BOUNDARY_CONDITION field with every kind (SOLID_WALL..FLUID) drawn per cell."""
    return np.random.default_rng(seed).integers(-4, 1, size=shape).astype(np.int32)


def test_generic_manager_2d_fill():
    """BOUNDARY_MANAGER_2D<TT>::SetBoundaryCondition on a random field with randomly mixed
    conditions per ghost cell: restatement equal to the reference's class, corners included."""
    geom = (4, 9, 9, 0.0, 1.0, 0.0, 1.0)
    a = Oracle2D(*geom, kind="port")
    b = Oracle2D(*geom, kind="reference")
    q = np.random.default_rng(1).uniform(0.5, 2.0, (a.ny + 6, a.nx + 6, 4))
    bc = random_conditions((a.ny + 6, a.nx + 6), 2)
    for o in (a, b):
        o.set_q(q)
        o.set_bc_field(bc)
        o.apply_bc()
    assert np.array_equal(a.get_q(), b.get_q())


def test_generic_manager_1d_fill_and_steps():
    n = 257
    geo = (5, 17, 0.5 / n, 1 - 0.5 / n)
    a, b = Oracle1D(*geo, kind="port"), Oracle1D(*geo, kind="reference")
    q = np.random.default_rng(3).uniform(0.5, 2.0, (n + 6, 3))
    for seed in range(4):
        bc = random_conditions(n + 6, 10 + seed)
        for o in (a, b):
            o.set_q(q)
            o.set_bc_field(bc)
            o.apply_bc()
        assert np.array_equal(a.get_q(), b.get_q()), seed
    # a run with periodic ends (left) and extrapolation (right)
    bc = np.full(n + 6, -2, np.int32)
    bc[:3] = -3
    for o in (a, b):
        o.init_riemann(0.5, (1.0, 0.0, 1.0), (0.125, 0.0, 0.1))
        o.set_bc_field(bc)
    t = 0.0
    for _ in range(20):
        oa, ob = a.step(1e-4, 0.5, t, 0.2), b.step(1e-4, 0.5, t, 0.2)
        assert np.array_equal(oa, ob)
        t += oa[0]
    assert np.array_equal(a.get_q(), b.get_q())


def test_generic_manager_2d_steps():
    """Steps with the generic manager (periodic in x, extrapolation in y, a SOLID_WALL corner
    block left alone): restatement equal to the reference."""
    geom = (4, 9, 9, 0.0, 10.0, 0.0, 10.0)
    a = Oracle2D(*geom, bc_kind=2, kind="port")
    b = Oracle2D(*geom, bc_kind=2, kind="reference")
    bc = np.full((a.ny + 6, a.nx + 6), -2, np.int32)
    bc[:, :3] = bc[:, -3:] = -3
    bc[:3, :3] = -4
    for o in (a, b):
        o.init_problem(2, 5.0, 5.0)
        o.set_bc_field(bc)
    t = 0.0
    for _ in range(4):
        oa, ob = a.step(1e-3, 0.4, t, 10.0), b.step(1e-3, 0.4, t, 10.0)
        assert np.array_equal(oa[:6], ob[:6])
        t += oa[0]
    assert np.array_equal(a.get_q(), b.get_q())
    assert np.array_equal(a.get_masks(), b.get_masks())


WT = (5, 13, 5, 0.0, 3.0, 0.0, 1.0)  # the wind tunnel's [0,3] x [0,1] on 193 x 65 nodes


def test_wind_tunnel_manager_calls():
    """BOUNDARY_MANAGER_WT: SetBoundaryCondition, the two bottom fills and BandingMask of the
    restatement equal the reference class's on a random field."""
    a = Oracle2D(*WT, bc_kind=5, kind="port")
    b = Oracle2D(*WT, bc_kind=5, kind="reference")
    q = np.random.default_rng(4).uniform(0.5, 2.0, (a.ny + 6, a.nx + 6, 4))
    for call in ("bc", 0, 1):
        for o in (a, b):
            o.set_q(q)
            if call == "bc":
                o.apply_bc()
            else:
                o.wt_call(call)
        assert np.array_equal(a.get_q(), b.get_q()), call
    m = np.zeros((5, a.ny + 6, a.nx + 6), np.uint8)
    for o in (a, b):
        o.set_masks(m)
        o.wt_call(2, 0)
    assert np.array_equal(a.get_masks(), b.get_masks())
    assert a.get_masks()[1].sum() > 0


def test_wind_tunnel_steps():
    """Mach 3 flow over the forward-facing step: 15 steps, restatement equal to the reference."""
    a = Oracle2D(*WT, bc_kind=5, kind="port")
    b = Oracle2D(*WT, bc_kind=5, kind="reference")
    for o in (a, b):
        o.init_problem(4, 0.0, 0.0)
    assert np.array_equal(a.get_q(), b.get_q())
    t = 0.0
    for k in range(15):
        oa, ob = a.step(1e-3, 0.4, t, 4.0), b.step(1e-3, 0.4, t, 4.0)
        assert np.array_equal(oa[:7], ob[:7]), (k, oa, ob)
        t += oa[0]
    assert np.array_equal(a.get_masks(), b.get_masks())
    assert np.array_equal(corner_free(a.get_q()), corner_free(b.get_q()))
