"""InterpolateAllGridEuler (dense field from the active points): the restatement against the
reference's own code on the CPU, and the CUDA path against the restatement on the GPU."""
import numpy as np
import pytest

import oracle
from oracle import Oracle2D

CASES = {
    "quad65": ((4, 9, 9, 0.0, 1.0, 0.0, 1.0), 0, 0, 0.5, 0.5, 1e-3, 0.4),
    "dmach": ((4, 17, 5, 0.0, 4.0, 0.0, 1.0), 1, 1, 1.4, 0.0, 1e-3, 0.5),
    "vortex": ((4, 9, 9, 0.0, 10.0, 0.0, 10.0), 2, 2, 5.0, 5.0, 1e-3, 0.4),
}


def stepped(make, case, n=3):
    geom, bc, prob, a, b, tol, cfl = CASES[case]
    o = make(geom, bc)
    o.init_problem(prob, a, b)
    t = 0.0
    for _ in range(n):
        t += o.step(tol, cfl, t, 10.0)[0]
    return o


@pytest.mark.parametrize("case", list(CASES))
def test_restatement_matches_reference(case):
    if not oracle.reference_available():
        pytest.skip("reference build absent")
    p = stepped(lambda g, bc: Oracle2D(*g, bc_kind=bc, kind="port"), case)
    r = stepped(lambda g, bc: Oracle2D(*g, bc_kind=bc, kind="reference"), case)
    assert np.array_equal(p.get_q()[3:-3, 3:-3], r.get_q()[3:-3, 3:-3])
    p.interpolate_all(0)
    r.interpolate_all(0)
    assert np.array_equal(p.get_q()[3:-3, 3:-3], r.get_q()[3:-3, 3:-3])


def test_dense_field_properties():
    """Values on mask0 are kept, every grid point ends with a positive density, and on the smooth
    vortex the dense field stays close to the analytic initial state."""
    geom, bc, prob, a, b, tol, cfl = CASES["vortex"]
    o = Oracle2D(*geom, bc_kind=bc, kind="port")
    o.init_problem(prob, a, b)
    exact = o.get_q()
    o.prepare(tol)
    o.manager(oracle.RR, 0)  # the between-steps state: values on mask0 only
    before = o.get_q()
    on = o.get_masks()[1, 3:-3, 3:-3].astype(bool)
    assert np.any(before[3:-3, 3:-3, 0][~on] == 0)
    o.interpolate_all(0)
    q = o.get_q()[3:-3, 3:-3]
    assert np.array_equal(q[on], before[3:-3, 3:-3][on])
    assert np.all(q[..., 0] > 0)
    err = np.abs(q - exact[3:-3, 3:-3]).max() / np.abs(exact[3:-3, 3:-3]).max()
    assert err < 5e-3, err


@pytest.mark.gpu
@pytest.mark.parametrize("case", list(CASES))
def test_gpu_matches_restatement(case, awcm_lib):
    p = stepped(lambda g, bc: Oracle2D(*g, bc_kind=bc, kind="port"), case)
    s = stepped(lambda g, bc: awcm_lib.AWCM2D(*g, bc_kind=bc), case)
    p.interpolate_all(0)
    s.interpolate_all(0)
    assert np.array_equal(s.get_q()[3:-3, 3:-3], p.get_q()[3:-3, 3:-3])


@pytest.mark.gpu
def test_gpu_dense_field_full_size(awcm_lib):
    """2049^2 four-quadrant state after two steps: dense field identical to the restatement's."""
    g = (7, 33, 33, 0.0, 1.0, 0.0, 1.0)
    p = Oracle2D(*g, bc_kind=0, kind="port")
    s = awcm_lib.AWCM2D(*g, bc_kind=0)
    t = 0.0
    for o in (p, s):
        o.init_problem(0, 0.5, 0.5)
    for _ in range(2):
        dt = p.step(1e-3, 0.4, t, 10.0)[0]
        assert s.step(1e-3, 0.4, t, 10.0)[0] == dt
        t += dt
    p.interpolate_all(0)
    s.interpolate_all(0)
    assert np.array_equal(s.get_q()[3:-3, 3:-3], p.get_q()[3:-3, 3:-3])
