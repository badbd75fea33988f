"""Failure handling on the GPU, with every failure made on the host.

* A NaN, an infinite momentum or a negative pressure written into the conserved field through the
  public state call makes the step return AWCM_ERR_NONFINITE (the CFL / Lax-Friedrichs speed scans
  flag the point); the instance is then restored from a state file and steps on bit for bit with
  the oracle.
* In a 1D batch, a poisoned instance stops with the flag while its neighbours keep stepping and
  stay identical to the oracle.
* The persistent PrepareEuler kernel's grid-barrier waits are given a limit of one poll (the
  test-only awcm2d_set_spin_limit), so they run out: the step returns AWCM_ERR_TIMEOUT instead
  of hanging, the device stays usable, and after the limit is restored the next step matches
  the oracle.
No failure here faults, traps or hangs the GPU: the waits are bounded and the data are only
values.
"""
import numpy as np
import pytest

from oracle import Oracle1D, Oracle2D
from oracle.state_format import read_state

pytestmark = pytest.mark.gpu

QUAD = (5, 9, 9, 0.0, 1.0, 0.0, 1.0)
TOL, CFL = 1e-3, 0.4
# A point of the coarsest grid (spacing 2^4 on the 129^2 grid): never thresholded, so it is in
# mask0 and hence in the CFL scan of mask3 at every step.
COARSE_MID = 64


def corner_free(q):
    keep = np.ones(q.shape[:2], bool)
    keep[:3, :3] = keep[:3, -3:] = keep[-3:, :3] = keep[-3:, -3:] = False
    return q[keep]


def stepped_pair(awcm, n):
    gpu = awcm.AWCM2D(*QUAD, bc_kind=0)
    ref = Oracle2D(*QUAD, bc_kind=0, kind="port")
    gpu.init_problem(0, 0.5, 0.5)
    ref.init_problem(0, 0.5, 0.5)
    t = 0.0
    for _ in range(n):
        o_g, o_r = gpu.step(TOL, CFL, t, 10.0), ref.step(TOL, CFL, t, 10.0)
        assert o_g[0] == o_r[0]
        t += o_r[0]
    return gpu, ref, t


def load_into_oracle(path, geom=QUAD, bc=0):
    r = read_state(path)
    o = Oracle2D(*geom, bc_kind=bc, kind="port")
    o.set_q(r["q"])
    o.set_masks(r["masks"])
    o.set_levels(r["levels"])
    return o, r["t"]


def assert_next_steps_match(gpu, ref, t, n=2):
    for _ in range(n):
        o_g, o_r = gpu.step(TOL, CFL, t, 10.0), ref.step(TOL, CFL, t, 10.0)
        assert o_g[0] == o_r[0] and np.array_equal(o_g[2:6], o_r[2:6])
        t += o_r[0]
    assert np.array_equal(gpu.get_masks(), ref.get_masks())
    assert np.array_equal(corner_free(gpu.get_q()), corner_free(ref.get_q()))


@pytest.mark.parametrize("poison", ["nan_density", "inf_momentum", "negative_pressure"])
def test_2d_nonfinite_state_is_reported_and_recoverable(tmp_path, awcm_lib, poison):
    gpu, _, t = stepped_pair(awcm_lib, 2)
    p = tmp_path / "good.bin"
    gpu.save_state(p, t, 2)
    q = gpu.get_q()
    jj = ii = COARSE_MID + 3
    if poison == "nan_density":
        q[jj, ii, 0] = np.nan
    elif poison == "inf_momentum":
        q[jj, ii, 1] = np.inf
    else:
        q[jj, ii, 3] = -1.0  # E < kinetic energy: p < 0, the sound speed is NaN
    gpu.set_q(q)
    with pytest.raises(awcm_lib.AwcmError) as ei:
        gpu.step(TOL, CFL, t, 10.0)
    assert ei.value.status == 5 and "non-finite" in str(ei.value)
    # the device and the instance stay usable: restore the saved state and continue
    import torch

    assert float(torch.ones(4, device="cuda").sum()) == 4.0
    tg, _ = gpu.load_state(p)
    ref, tr = load_into_oracle(p)
    assert tg == tr == t
    assert_next_steps_match(gpu, ref, t)


def test_2d_advance_stops_at_nonfinite_step(awcm_lib):
    gpu, _, t = stepped_pair(awcm_lib, 1)
    q = gpu.get_q()
    q[COARSE_MID + 3, COARSE_MID + 3, 0] = np.nan
    gpu.set_q(q)
    with pytest.raises(awcm_lib.AwcmError) as ei:
        gpu.advance(TOL, CFL, t, 10.0, 5)
    assert ei.value.status == 5


def test_1d_batch_isolates_a_nonfinite_instance(awcm_lib):
    n = 257
    b = awcm_lib.AWCM1DBatch([5, 5, 5], 17, 0.5 / n, 1 - 0.5 / n)
    refs = []
    for k in range(3):
        b.init_riemann(k, 0.5, (1.0, 0.0, 1.0), (0.125, 0.0, 0.1))
        o = Oracle1D(5, 17, 0.5 / n, 1 - 0.5 / n, kind="port")
        o.init_riemann(0.5, (1.0, 0.0, 1.0), (0.125, 0.0, 0.1))
        refs.append(o)
    q = b.get_q(1)
    q[n // 2 + 3, 0] = np.nan  # point 128: a point of the coarsest grid
    b.set_q(1, q)
    b.set_run(1e-4, 0.5, 0.0, 0.2)
    b.steps(4)
    s1 = b.status(1)
    assert s1[14] == 5 and s1[3] == 1 and s1[4] == 1, s1  # flagged on its first step, then stopped
    with pytest.raises(awcm_lib.AwcmError) as ei:
        b.check_finite(1)
    assert ei.value.status == 5
    t = 0.0
    for _ in range(4):
        dt = refs[0].step(1e-4, 0.5, t, 0.2)[0]
        refs[2].step(1e-4, 0.5, t, 0.2)
        t += dt
    for k in (0, 2):
        s = b.status(k)
        assert s[14] == 0 and s[4] == 4
        assert np.array_equal(b.get_q(k), refs[k].get_q())
        assert np.array_equal(b.get_masks(k), refs[k].get_masks())
    # set_run clears the flag; with a finite state the instance steps again
    good = Oracle1D(5, 17, 0.5 / n, 1 - 0.5 / n, kind="port")
    good.init_riemann(0.5, (1.0, 0.0, 1.0), (0.125, 0.0, 0.1))
    b.set_q(1, good.get_q())
    b.set_masks(1, good.get_masks())
    b.set_levels(1, good.get_levels())
    b.set_run(1e-4, 0.5, 0.0, 0.2)
    b.steps(1)
    assert b.status(1)[14] == 0
    good.step(1e-4, 0.5, 0.0, 0.2)
    assert np.array_equal(b.get_q(1), good.get_q())


def test_persistent_prepare_barrier_timeout(tmp_path, awcm_lib):
    gpu, _, t = stepped_pair(awcm_lib, 2)
    p = tmp_path / "good.bin"
    gpu.save_state(p, t, 2)
    gpu.set_prepare_mode(0)
    gpu.set_spin_limit(1)
    with pytest.raises(awcm_lib.AwcmError) as ei:
        gpu.step(TOL, CFL, t, 10.0)
    assert ei.value.status == 4 and "barrier" in str(ei.value)
    import torch

    assert float(torch.arange(8, device="cuda", dtype=torch.float64).sum()) == 28.0
    gpu.set_spin_limit(0)
    gpu.load_state(p)
    ref, _ = load_into_oracle(p)
    assert_next_steps_match(gpu, ref, t)
