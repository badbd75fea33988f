"""Frozen-mask run and discrete adjoint of the 2D path on the GPU.

* The frozen-mask forward (no PrepareEuler / residue removal, fixed dt, LF speeds recorded or
  replayed) is bit-identical to the CPU restatement and to the reference's own code, and its
  central differences equal the reference's (tests/golden/adjoint_vortex65.npz) bit for bit.
* The adjoint's directional derivatives agree with FP64 central finite differences (16 seeded
  directions of unit L2 norm) to 1e-6 relative in the differentiable mode (WENO-Z eps = 1e-6 and
  tau = sqrt((b0-b2)^2 + delta^2), delta = 1e-6): with h = 1e-6 on the fixture grid (65^2,
  10 steps), and on the 513^2 / 200-step gradient workload with h = 1e-5.  There a unit direction
  spreads over 10^6 values (1e-9 each at h = 1e-6), and the rounding of the 200-step run moves the
  loss difference by ~6e-15, i.e. ~3e-9 on a directional derivative of 2e-4: differences at
  h = 1e-6 of the weakest directions scatter by up to 1.5e-5 relative around the h = 1e-5 value,
  which itself agrees with the adjoint to better than 5e-7 in all 16 directions.
* Against the reference solver's own central differences (eps = 1e-6, exact |b0 - b2|, which the
  reference cannot smooth) the agreement is bounded by the differences' own noise: with |.| the
  map has kinks, and central differences at h = 1e-6 and 1e-7 of the same direction differ by
  up to 7e-5 relative (CPU restatement, 16 directions); the bound used is 2e-4.
* Checkpoint intervals (every step, sqrt(N), keep-all) give the same gradient.
* The torch.autograd.Function harness passes torch.autograd.gradcheck (fast mode).
"""
import os

import numpy as np
import pytest

import oracle
from oracle import Oracle2D

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
FD_REL_TOL = 1e-6
REF_FD_REL_TOL = 2e-4
EPS_DIFF = 1e-6    # WENO-Z epsilon of the differentiable mode
DELTA_DIFF = 1e-6  # smoothing of |b0 - b2| in the differentiable mode


def fixture():
    return dict(np.load(os.path.join(GOLDEN, "adjoint_vortex65.npz")))


def small_solver(awcm, g):
    nl, nxc = int(g["params"][0]), int(g["params"][1])
    s = awcm.AWCM2D(nl, nxc, nxc, 0.0, 10.0, 0.0, 10.0, bc_kind=awcm.BC_PERIODIC)
    return s


def prepared_small(awcm):
    """GPU instance of the fixture case after one PrepareEuler on the seeded initial state."""
    from awcm import gradient as G

    g = fixture()
    s = small_solver(awcm, g)
    q0 = G.vortex_bumps(s)
    s.set_q(q0)
    s.prepare(float(g["params"][2]))
    return s, g


def replay_q(s, q, dt, n):
    s.set_q(q)
    s.frozen_run(0.0, dt, n, replay=True)
    return s.get_q()


def test_prepared_state_matches_fixture(awcm_lib):
    s, g = prepared_small(awcm_lib)
    assert np.array_equal(s.get_q(), g["q"])
    assert np.array_equal(s.get_masks(), g["masks"])
    assert np.array_equal(s.get_levels(), g["levels"])


@pytest.mark.parametrize("eps,delta", [(1e-40, 0.0), (EPS_DIFF, 0.0), (EPS_DIFF, DELTA_DIFF)])
def test_frozen_run_bitexact_vs_checkers(awcm_lib, eps, delta):
    """Recording run: end state and LF-speed tape equal the restatement's (and the reference's,
    when its build is present and the mode is one it has) bit for bit."""
    s, g = prepared_small(awcm_lib)
    s.set_wenoz(eps, delta)
    nl, nxc, steps = int(g["params"][0]), int(g["params"][1]), int(g["params"][4])
    dt = float(g["dt"])
    qp = s.get_q()
    s.frozen_run(0.0, dt, steps)
    q_gpu, tape_gpu = s.get_q(), s.get_alpha_tape(steps)
    kinds = ["port"] + (["reference"] if oracle.reference_available() and delta == 0 else [])
    for kind in kinds:
        o = Oracle2D(nl, nxc, nxc, 0.0, 10.0, 0.0, 10.0, bc_kind=2, kind=kind)
        o.set_q(qp)
        o.set_masks(g["masks"])
        o.set_levels(g["levels"])
        o.set_wenoz(eps, delta)
        o.set_freeze(1)
        tape = np.zeros_like(tape_gpu)
        t = 0.0
        for k in range(steps):
            o.step(0.0, 1.0, t, 1e300, dt, tape[k])
            t += dt
        assert np.array_equal(tape, tape_gpu), kind
        qo = o.get_q()
        inner = (slice(3, -3), slice(3, -3))
        assert np.array_equal(q_gpu[inner], qo[inner]), kind
    if eps == EPS_DIFF and delta == 0:
        assert np.array_equal(tape_gpu, g["tape"])
        assert np.array_equal(q_gpu[3:-3, 3:-3], g["q_end"][3:-3, 3:-3])


def test_gpu_finite_differences_equal_reference(awcm_lib):
    """Central differences of the GPU frozen replay equal the reference's bit for bit."""
    from awcm import gradient as G

    s, g = prepared_small(awcm_lib)
    s.set_wenoz(EPS_DIFF)
    _, _, _, _, steps, n_dirs, seed, h = g["params"]
    steps, n_dirs, seed = int(steps), int(n_dirs), int(seed)
    s.set_alpha_tape(g["tape"])
    dirs = G.unit_directions(g["q"].shape, n_dirs, seed)
    for k in range(n_dirs):
        a = replay_q(s, g["q"] + h * dirs[k], float(g["dt"]), steps)
        b = replay_q(s, g["q"] - h * dirs[k], float(g["dt"]), steps)
        assert G.loss_difference(a, b, g["target"], G.active_points(g["masks"])) / (2 * h) == g["fd"][k], k


def directional_errors(grad, dirs, fd):
    ad = np.array([float(np.sum(grad * d)) for d in dirs])
    return ad, np.abs(ad - fd) / np.abs(fd)


def test_adjoint_vs_reference_directional_gradient(awcm_lib):
    """Adjoint directional derivatives against the reference solver's central differences
    (WENO-Z eps 1e-6, exact |b0 - b2|)."""
    from awcm import gradient as G

    s, g = prepared_small(awcm_lib)
    s.set_wenoz(EPS_DIFF)
    _, _, _, _, steps, n_dirs, seed, h = g["params"]
    s.set_alpha_tape(g["tape"])
    loss, grad, info = s.adjoint(0.0, float(g["dt"]), int(steps), g["target"], replay=True)
    dirs = G.unit_directions(g["q"].shape, int(n_dirs), int(seed))
    ad, rel = directional_errors(grad, dirs, g["fd"])
    print("adjoint vs reference differences: max rel %.2e" % rel.max())
    assert rel.max() <= REF_FD_REL_TOL, (rel, ad, g["fd"])
    # loss of the replayed run, same value as the recording run's
    assert loss == pytest.approx(G.loss(g["q_end"], g["target"], G.active_points(g["masks"])), rel=1e-13)
    assert np.all(grad[:3] == 0) and np.all(grad[-3:] == 0) and np.all(grad[:, :3] == 0) and np.all(grad[:, -3:] == 0)


def test_adjoint_vs_differences_differentiable_mode(awcm_lib):
    """Differentiable mode on the fixture grid: 16 directions, h = 1e-6, GPU frozen replay."""
    from awcm import gradient as G

    s, g = prepared_small(awcm_lib)
    s.set_wenoz(EPS_DIFF, DELTA_DIFF)
    _, _, _, _, steps, n_dirs, seed, h = g["params"]
    steps, dt = int(steps), float(g["dt"])
    s.set_q(g["q"])
    loss, grad, info = s.adjoint(0.0, dt, steps, g["target"])
    dirs = G.unit_directions(g["q"].shape, int(n_dirs), int(seed))
    act = G.active_points(g["masks"])
    fd = np.array([G.loss_difference(replay_q(s, g["q"] + h * d, dt, steps), replay_q(s, g["q"] - h * d, dt, steps),
                                     g["target"], act) / (2 * h) for d in dirs])
    ad, rel = directional_errors(grad, dirs, fd)
    print("adjoint vs differences (differentiable mode, 65^2): max rel %.2e" % rel.max())
    assert rel.max() <= FD_REL_TOL, (rel, ad, fd)


def test_checkpoint_intervals_agree(awcm_lib):
    s, g = prepared_small(awcm_lib)
    s.set_wenoz(EPS_DIFF)
    steps, dt = int(g["params"][4]), float(g["dt"])
    s.set_alpha_tape(g["tape"])
    grads = []
    for every in (1, 3, 0, steps):
        s.set_q(g["q"])
        loss, grad, info = s.adjoint(0.0, dt, steps, g["target"], checkpoint_every=every, replay=True)
        grads.append((loss, grad, info))
        # the state is left at the end of the forward run
        assert np.array_equal(s.get_q()[3:-3, 3:-3], g["q_end"][3:-3, 3:-3])
    ref_loss, ref_grad, _ = grads[-1]
    scale = np.abs(ref_grad).max()
    for loss, grad, info in grads[:-1]:
        assert loss == ref_loss
        assert np.abs(grad - ref_grad).max() <= 1e-12 * scale, info
    assert grads[2][2]["checkpoint_every"] == int(np.ceil(np.sqrt(steps)))


def test_adjoint_recording_equals_replay(awcm_lib):
    """mode 1 (record during the adjoint's forward) and mode 2 (replay) give the same result."""
    s, g = prepared_small(awcm_lib)
    s.set_wenoz(EPS_DIFF)
    steps, dt = int(g["params"][4]), float(g["dt"])
    s.set_q(g["q"])
    l1, g1, _ = s.adjoint(0.0, dt, steps, g["target"])
    assert np.array_equal(s.get_alpha_tape(steps), g["tape"])
    s.set_q(g["q"])
    l2, g2, _ = s.adjoint(0.0, dt, steps, g["target"], replay=True)
    assert l1 == l2
    assert np.abs(g1 - g2).max() <= 1e-12 * np.abs(g2).max()


def test_gradient_workload_full_size(awcm_lib):
    """513^2 periodic vortex + bumps, 200 frozen steps, sqrt(N) checkpoints: 16 seeded unit
    directions against central differences of the GPU frozen replay (h = 1e-5, the smallest step
    above the run's rounding floor)."""
    from awcm import gradient as G

    s = awcm_lib.AWCM2D(6, 17, 17, 0.0, 10.0, 0.0, 10.0, bc_kind=awcm_lib.BC_PERIODIC)
    assert (s.nx, s.ny) == (513, 513)
    q0 = G.vortex_bumps(s)
    target = G.target_density(s)
    dt = G.stable_dt(q0, 10.0 / 512)
    s.set_q(q0)
    s.prepare(1e-3)
    s.set_wenoz(EPS_DIFF, DELTA_DIFF)
    qp = s.get_q()
    n = 200
    loss, grad, info = s.adjoint(0.0, dt, n, target)
    assert info["checkpoint_every"] == 15
    assert np.isfinite(loss) and np.isfinite(grad).all()
    h = 1e-5
    act = G.active_points(s.get_masks())
    dirs = G.unit_directions(qp.shape, 16, 11)
    fd = []
    for d in dirs:
        a = replay_q(s, qp + h * d, dt, n)
        b = replay_q(s, qp - h * d, dt, n)
        fd.append(G.loss_difference(a, b, target, act) / (2 * h))
    ad, rel = directional_errors(grad, dirs, np.array(fd))
    print("full-size adjoint: loss %.6e fwd %.1f ms rev %.1f ms max rel %.2e" %
          (loss, info["forward_ms"], info["reverse_ms"], rel.max()))
    assert rel.max() <= FD_REL_TOL, (rel, ad, fd)


def test_torch_autograd_harness(awcm_lib):
    import torch

    from awcm import gradient as G

    s = awcm_lib.AWCM2D(3, 9, 9, 0.0, 10.0, 0.0, 10.0, bc_kind=awcm_lib.BC_PERIODIC)
    q0 = G.vortex_bumps(s)
    target = G.target_density(s)
    dt = G.stable_dt(q0, 10.0 / (s.nx - 1))
    s.set_q(q0)
    s.prepare(1e-3)
    s.set_wenoz(EPS_DIFF, DELTA_DIFF)
    qp = s.get_q()
    s.frozen_run(0.0, dt, 4)  # records the LF-speed tape the harness replays
    F = G.frozen_loss_function()
    x = torch.from_numpy(qp).requires_grad_(True)
    loss = F.apply(x, s, target, 0.0, dt, 4, 0)
    loss.backward()
    assert x.grad is not None and torch.isfinite(x.grad).all()
    assert torch.autograd.gradcheck(lambda y: F.apply(y, s, target, 0.0, dt, 4, 0), (x,), eps=1e-6, atol=1e-8,
                                    rtol=1e-5, fast_mode=True)


@pytest.mark.parametrize("bc", [0, 1, 3])
def test_adjoint_boundary_folds(awcm_lib, bc):
    """Transposed boundary fills of the transmissive, double-Mach and wall managers: the adjoint
    against central differences (h = 1e-6), differentiable mode.  The transmissive and wall
    managers run on the vortex + bumps state (bound 1e-6); the double-Mach manager on its own
    initial state (129 x 33 nodes, 6 steps at a quarter of the CFL limit, target 1.01 rho0), whose
    shock leaves central differences at h = 1e-6 and 1e-7 up to 1.5e-6 apart (CPU restatement),
    so the bound there is 2e-5."""
    from awcm import gradient as G

    if bc == 1:
        s = awcm_lib.AWCM2D(4, 17, 5, 0.0, 4.0, 0.0, 1.0, bc_kind=1)
        s.init_problem(awcm_lib.PROBLEM_DOUBLE_MACH, 1.4, 0.0)
        q0 = s.get_q()
        target = 1.01 * q0[3:-3, 3:-3, 0]
        dt = 0.25 * (4.0 / (s.nx - 1)) / 22.0
        tol_rel = 2e-5
    else:
        s = awcm_lib.AWCM2D(4, 9, 9, 0.0, 10.0, 0.0, 10.0, bc_kind=bc)
        q0, target = G.vortex_bumps(s), G.target_density(s)
        dt = G.stable_dt(q0, 10.0 / (s.nx - 1))
        tol_rel = FD_REL_TOL
    s.set_q(q0)
    s.prepare(1e-3)
    s.set_wenoz(EPS_DIFF, DELTA_DIFF)
    qp = s.get_q()
    n = 6
    loss, grad, _ = s.adjoint(0.0, dt, n, target)
    act = G.active_points(s.get_masks())
    dirs = G.unit_directions(qp.shape, 8, 5)
    h = 1e-6
    fd = np.array([G.loss_difference(replay_q(s, qp + h * d, dt, n), replay_q(s, qp - h * d, dt, n), target, act)
                   / (2 * h) for d in dirs])
    ad, rel = directional_errors(grad, dirs, fd)
    print(f"adjoint vs differences, boundary kind {bc}: max rel {rel.max():.2e}")
    assert rel.max() <= tol_rel, (rel, ad, fd)
