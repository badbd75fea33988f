"""Seeded synthetic workloads of the benchmark configurations (no dataset is involved)."""
from __future__ import annotations

import numpy as np

SEED = 20261203


def shock_tubes(n: int = 512, seed: int = SEED, jmin: int = 4, jmax=(8, 13)):
    """The uneven shock-tube batch: rho_L, rho_R, p_L, p_R log-uniform in [0.1, 10], u_L, u_R uniform
    in [-1, 1], interface uniform in [0.3, 0.7], Jmax uniform in {8..13}, Jmin 4 (17 coarse nodes),
    cell-centred nodes on [0, 1].  Returns a list of dicts."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        J = int(rng.integers(jmax[0], jmax[1] + 1))
        L = J - jmin + 1
        nx = 16 * 2 ** (L - 1) + 1
        rl, rr, pl, pr = (10.0 ** rng.uniform(-1, 1, size=4)).tolist()
        ul, ur = rng.uniform(-1, 1, size=2).tolist()
        xi = float(rng.uniform(0.3, 0.7))
        out.append(dict(jmax=J, num_levels=L, nx_coarse=2 ** jmin + 1, nx=nx, x_min=0.5 / nx, x_max=1 - 0.5 / nx,
                        x_interface=xi, left=(rl, ul, pl), right=(rr, ur, pr)))
    return out


def make_batch(awcm, tubes, scheme=0):
    b = awcm.AWCM1DBatch([t["num_levels"] for t in tubes], [t["nx_coarse"] for t in tubes],
                         [t["x_min"] for t in tubes], [t["x_max"] for t in tubes], scheme=scheme)
    for k, t in enumerate(tubes):
        b.init_riemann(k, t["x_interface"], t["left"], t["right"])
    return b
