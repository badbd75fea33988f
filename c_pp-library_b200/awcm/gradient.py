"""Gradient workload of the frozen-mask adjoint and its torch.autograd harness.

Workload (isentropic vortex with seeded density bumps on the periodic square [0,10]^2):
  * the vortex of ISENTROPIC_VORTEX_ADVECTION::Initialize
    (Problems/2D/PROBLEM_ISENTROPIC_VORTEX_ADVECTION.h:38-64), strength 5, radius 1, gamma 1.4,
    centred at (5, 5);
  * plus 16 Gaussian density bumps rho += a exp(-|x - c|^2 / w^2) with a ~ U[0, 0.05],
    w ~ U[0.3, 1], c ~ U[0,10]^2 (distances taken periodically), velocity and pressure kept;
  * target = the density of the same construction from a second seed;
  * loss = 1/2 sum over the active points (mask0 of the frozen masks) of (rho(t_end) - target)^2
    after n frozen-mask RK3 steps; points outside the masks hold no solution value (PrepareEuler
    leaves them at zero).

``FrozenLoss`` wraps ``AWCM2D.adjoint`` as a torch.autograd.Function: its forward runs the frozen
run with the LF speeds replayed from the solver's tape and returns the loss, its backward hands
back the adjoint gradient.  It exists to let torch.autograd.gradcheck compare the hand-written
adjoint with finite differences; nothing else uses it.
"""
from __future__ import annotations

import numpy as np

GAMMA = 1.4
VORTEX_SEED = 20261203
TARGET_SEED = 20261204


def bumps(seed: int, n: int = 16):
    """(amplitude, width, cx, cy) of n seeded Gaussian density bumps."""
    rng = np.random.default_rng(seed)
    a = rng.uniform(0.0, 0.05, n)
    w = rng.uniform(0.3, 1.0, n)
    c = rng.uniform(0.0, 10.0, (n, 2))
    return a, w, c[:, 0], c[:, 1]


def add_bumps(q: np.ndarray, x_min: float, y_min: float, dx: float, dy: float, seed: int,
              period: float = 10.0) -> np.ndarray:
    """Adds the seeded density bumps to a conserved state (Ny+6, Nx+6, 4), ghosts included,
    keeping velocity and pressure."""
    q = np.array(q, dtype=np.float64, copy=True)
    ny, nx = q.shape[0] - 6, q.shape[1] - 6
    x = x_min + (np.arange(nx + 6) - 3) * dx
    y = y_min + (np.arange(ny + 6) - 3) * dy
    X, Y = np.meshgrid(x, y)
    rho = q[..., 0]
    u, v = q[..., 1] / rho, q[..., 2] / rho
    p = (GAMMA - 1) * (q[..., 3] - 0.5 * (q[..., 1] ** 2 + q[..., 2] ** 2) / rho)
    drho = np.zeros_like(rho)
    for a, w, cx, cy in zip(*bumps(seed)):
        ddx = np.abs(X - cx)
        ddy = np.abs(Y - cy)
        ddx = np.minimum(ddx, period - ddx)
        ddy = np.minimum(ddy, period - ddy)
        drho += a * np.exp(-(ddx ** 2 + ddy ** 2) / (w * w))
    rho2 = rho + drho
    q[..., 0] = rho2
    q[..., 1] = rho2 * u
    q[..., 2] = rho2 * v
    q[..., 3] = p / (GAMMA - 1) + 0.5 * rho2 * (u * u + v * v)
    return q


def vortex_bumps(solver, seed: int = VORTEX_SEED) -> np.ndarray:
    """Initial state of the gradient workload on `solver` (anything with init_problem/get_q and
    nx, ny over [0,10]^2): returned, not set."""
    solver.init_problem(2, 5.0, 5.0)
    q = solver.get_q()
    d = 10.0 / (solver.nx - 1)
    return add_bumps(q, 0.0, 0.0, d, 10.0 / (solver.ny - 1), seed)


def target_density(solver, seed: int = TARGET_SEED) -> np.ndarray:
    """Ny x Nx target density: the same construction from a second seed."""
    q = vortex_bumps(solver, seed)
    return np.ascontiguousarray(q[3:-3, 3:-3, 0])


def stable_dt(q: np.ndarray, dx: float, cfl: float = 0.4) -> float:
    """cfl dx / max(|u|+c + |v|+c) over the grid points, rounded down to 3 significant digits."""
    g = q[3:-3, 3:-3]
    rho = g[..., 0]
    u, v = g[..., 1] / rho, g[..., 2] / rho
    p = (GAMMA - 1) * (g[..., 3] - 0.5 * rho * (u * u + v * v))
    c = np.sqrt(GAMMA * p / rho)
    dt = cfl * dx / float(np.max(np.abs(u) + c + np.abs(v) + c))
    e = np.floor(np.log10(dt)) - 2
    return float(np.floor(dt / 10 ** e) * 10 ** e)


def unit_directions(shape, count: int, seed: int) -> np.ndarray:
    """count seeded directions of unit L2 norm over the grid points of a (Ny+6, Nx+6, 4) state
    (zero on the ghost ring, which the boundary fill overwrites)."""
    rng = np.random.default_rng(seed)
    out = np.zeros((count,) + tuple(shape))
    for k in range(count):
        d = rng.standard_normal((shape[0] - 6, shape[1] - 6, shape[2]))
        out[k, 3:-3, 3:-3] = d / np.linalg.norm(d)
    return out


def active_points(masks: np.ndarray) -> np.ndarray:
    """Ny x Nx bool of mask0 from the (5, Ny+6, Nx+6) mask planes (mask_temp, mask0..mask3)."""
    return masks[1, 3:-3, 3:-3].astype(bool)


def loss(q: np.ndarray, target: np.ndarray, active: np.ndarray) -> float:
    a = (q[3:-3, 3:-3, 0] - target)[active]
    return float(0.5 * np.sum(a * a))


def loss_difference(q_plus: np.ndarray, q_minus: np.ndarray, target: np.ndarray, active: np.ndarray) -> float:
    """L(q+) - L(q-) of L = 1/2 sum over the active points of (rho - target)^2, summed as
    1/2 (a+ - a-)(a+ + a-) per point to keep the cancellation out of the difference."""
    ap = (q_plus[3:-3, 3:-3, 0] - target)[active]
    am = (q_minus[3:-3, 3:-3, 0] - target)[active]
    return float(0.5 * np.sum((ap - am) * (ap + am)))


def _torch_function():
    import torch

    class FrozenLoss(torch.autograd.Function):
        """loss = FrozenLoss.apply(q0, solver, target, t0, dt, n_steps, checkpoint_every)."""

        @staticmethod
        def forward(ctx, q0, solver, target, t0, dt, n_steps, checkpoint_every=0):
            solver.set_q(q0.detach().cpu().numpy())
            loss, grad, _ = solver.adjoint(t0, dt, n_steps, target, checkpoint_every, replay=True)
            ctx.save_for_backward(torch.from_numpy(grad))
            return torch.tensor(loss, dtype=torch.float64)

        @staticmethod
        def backward(ctx, g):
            (grad,) = ctx.saved_tensors
            return g * grad, None, None, None, None, None, None

    return FrozenLoss


_FROZEN_LOSS = None


def frozen_loss_function():
    """The torch.autograd.Function over AWCM2D.adjoint (built on first use; imports torch)."""
    global _FROZEN_LOSS
    if _FROZEN_LOSS is None:
        _FROZEN_LOSS = _torch_function()
    return _FROZEN_LOSS
