"""The wind-tunnel manager (BOUNDARY_MANAGER_WT, Problems/2D/PROBLEM_WINDTUNNEL.h:52-222) on the GPU
against the reference's own class (through the harness) and the CPU restatement: its standard fill,
its two per-direction bottom fills and its BandingMask on a random field, and the Mach 3 flow over
the forward-facing step stepped with the per-direction fills, bit for bit."""
import numpy as np
import pytest

import oracle
from oracle import Oracle2D

pytestmark = pytest.mark.gpu

WT = (5, 13, 5, 0.0, 3.0, 0.0, 1.0)  # [0,3] x [0,1] on 193 x 65 nodes; step corner (38, 12)


def kinds():
    return ["port", "reference"] if oracle.reference_available() else ["port"]


def corner_free(q):
    keep = np.ones(q.shape[:2], bool)
    keep[:3, :3] = keep[:3, -3:] = keep[-3:, :3] = keep[-3:, -3:] = False
    return q[keep]


def test_manager_calls(awcm_lib):
    gpu = awcm_lib.AWCM2D(*WT, bc_kind=awcm_lib.BC_WIND_TUNNEL)
    q = np.random.default_rng(4).uniform(0.5, 2.0, (gpu.ny + 6, gpu.nx + 6, 4))
    for call in ("bc", "x", "y"):
        gpu.set_q(q)
        if call == "bc":
            gpu.apply_bc()
        else:
            gpu.wt_set_bottom(call == "x", call == "y")
        for kind in kinds():
            o = Oracle2D(*WT, bc_kind=5, kind=kind)
            o.set_q(q)
            if call == "bc":
                o.apply_bc()
            else:
                o.wt_call(0 if call == "x" else 1)
            assert np.array_equal(gpu.get_q(), o.get_q()), (call, kind)
    m = np.zeros((5, gpu.ny + 6, gpu.nx + 6), np.uint8)
    gpu.set_masks(m)
    gpu.manager(awcm_lib.BAND, 0)
    for kind in kinds():
        o = Oracle2D(*WT, bc_kind=5, kind=kind)
        o.set_masks(m)
        o.wt_call(2, 0)
        assert np.array_equal(gpu.get_masks()[1], o.get_masks()[1]), kind
    with pytest.raises(awcm_lib.AwcmError):
        gpu.wt_set_bottom(True, True)


@pytest.mark.parametrize("steps", [15, 60])
def test_steps_over_the_step(awcm_lib, steps):
    gpu = awcm_lib.AWCM2D(*WT, bc_kind=awcm_lib.BC_WIND_TUNNEL)
    gpu.init_problem(awcm_lib.PROBLEM_WIND_TUNNEL, 0.0, 0.0)
    refs = []
    for kind in kinds() if steps == 15 else ["port"]:
        o = Oracle2D(*WT, bc_kind=5, kind=kind)
        o.init_problem(4, 0.0, 0.0)
        refs.append(o)
    assert np.array_equal(gpu.get_q(), refs[0].get_q())
    t = 0.0
    for k in range(steps):
        o_g = gpu.step(1e-3, 0.4, t, 4.0)
        for o in refs:
            o_r = o.step(1e-3, 0.4, t, 4.0)
            assert o_g[0] == o_r[0] and np.array_equal(o_g[2:6], o_r[2:6]), (k, o.kind, o_g, o_r)
        t += o_g[0]
    for o in refs:
        assert np.array_equal(gpu.get_masks(), o.get_masks()), o.kind
        assert np.array_equal(corner_free(gpu.get_q()), corner_free(o.get_q())), o.kind
    with pytest.raises(awcm_lib.AwcmError, match="wind-tunnel"):
        gpu.frozen_run(t, 1e-3, 2)
