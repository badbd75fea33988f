"""Generates the golden fixtures of tests/golden/ from the reference's own code.

The reference (doseongju/C_pp-library) ships no tests, fixtures or known-answer vectors, so the
fixtures here are outputs of the reference itself: its headers compiled from the reference tree by
oracle/Makefile behind oracle/ref_harness_{1d,2d}.cpp, run on small seeded/deterministic cases.
Only this script touches the reference build; the tests replay the fixtures against the CPU
restatement (everywhere) and the CUDA path (on a GPU).

    make -C oracle ref && python tests/golden/make_golden.py [1d] [2d] [adjoint]
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "c_pp-library_b200"))

import oracle  # noqa: E402

N_SOD = 1025
SOD_1D = dict(num_levels=7, nx_coarse=17, x_min=0.5 / N_SOD, x_max=1 - 0.5 / N_SOD)

CASES_2D = {
    # name: (num_levels, nx_coarse, ny_coarse, domain, bc_kind, problem, a, b, tol, cfl, steps)
    "quad65": (4, 9, 9, (0.0, 1.0, 0.0, 1.0), 0, 0, 0.5, 0.5, 1e-3, 0.4, 6),
    "quad129_refsplit": (5, 9, 9, (0.0, 1.0, 0.0, 1.0), 0, 0, 0.8, 0.8, 1e-4, 0.5, 4),
    "dmach129x33": (4, 17, 5, (0.0, 4.0, 0.0, 1.0), 1, 1, 1.4, 0.0, 1e-3, 0.5, 5),
    "vortex65": (4, 9, 9, (0.0, 10.0, 0.0, 10.0), 2, 2, 5.0, 5.0, 1e-3, 0.4, 5),
}


def gen_1d():
    out = {}
    for scheme, tag in ((0, "wenoz"), (1, "weno5")):
        r = oracle.Oracle1D(**SOD_1D, scheme=scheme, kind="reference")
        r.init_riemann(0.5, (1.0, 0.0, 1.0), (0.125, 0.0, 0.1))
        steps = []
        t = 0.0
        for _ in range(10):
            o = r.step(1e-4, 0.5, t, 0.2)
            steps.append(o)
            t += o[0]
        out[f"sod1d_{tag}_10"] = dict(q=r.get_q(), masks=r.get_masks(), levels=r.get_levels(), steps=np.array(steps),
                                      t=t, scheme=scheme)
    r = oracle.Oracle1D(**SOD_1D, scheme=0, kind="reference")
    r.init_riemann(0.5, (1.0, 0.0, 1.0), (0.125, 0.0, 0.1))
    n, t, upd = r.run(1e-4, 0.5, 0.2)
    out["sod1d_wenoz_full"] = dict(q=r.get_q(), masks=r.get_masks(), levels=r.get_levels(),
                                   run=np.array([n, t, upd]), scheme=0)
    # uneven batch members: seeded Riemann states, short runs
    rng = np.random.default_rng(20261203)
    for k, L in enumerate((5, 6, 8)):
        nx = 16 * 2 ** (L - 1) + 1
        xi = rng.uniform(0.3, 0.7)
        left = (10 ** rng.uniform(-1, 1), rng.uniform(-1, 1), 10 ** rng.uniform(-1, 1))
        right = (10 ** rng.uniform(-1, 1), rng.uniform(-1, 1), 10 ** rng.uniform(-1, 1))
        r = oracle.Oracle1D(L, 17, 0.5 / nx, 1 - 0.5 / nx, kind="reference")
        r.init_riemann(xi, left, right)
        n, t, upd = r.run(1e-4, 0.5, 0.02)
        out[f"tube{k}_L{L}"] = dict(q=r.get_q(), masks=r.get_masks(), levels=r.get_levels(),
                                    run=np.array([n, t, upd]), geom=np.array([L, 17, 0.5 / nx, 1 - 0.5 / nx]),
                                    riemann=np.array([xi, *left, *right]))
    return out


def gen_2d():
    out = {}
    for name, (nl, nxc, nyc, dom, bc, prob, a, b, tol, cfl, steps) in CASES_2D.items():
        r = oracle.Oracle2D(nl, nxc, nyc, *dom, bc_kind=bc, kind="reference")
        r.init_problem(prob, a, b)
        q0 = r.get_q()
        rec = []
        t = 0.0
        for _ in range(steps):
            o = r.step(tol, cfl, t, 10.0)
            rec.append(o)
            t += o[0]
        out[name] = dict(q0=q0, q=r.get_q(), masks=r.get_masks(), levels=r.get_levels()[:3], steps=np.array(rec),
                         params=np.array([nl, nxc, nyc, *dom, bc, prob, a, b, tol, cfl, steps]))
    return out


# Gradient workload on a small grid: vortex + seeded density bumps on periodic [0,10]^2, frozen
# masks from one PrepareEuler, WENO-Z eps 1e-6 (the differentiable mode), fixed dt.
ADJ_CASE = dict(num_levels=4, nx_coarse=9, tol=1e-3, eps=1e-6, steps=10, n_dirs=16, dir_seed=7, h=1e-6)


def frozen_replay(kind, q, masks, levels, tape, dt, eps, nl, nxc):
    r = oracle.Oracle2D(nl, nxc, nxc, 0.0, 10.0, 0.0, 10.0, bc_kind=2, kind=kind)
    r.set_q(q)
    r.set_masks(masks)
    r.set_levels(levels)
    r.set_wenoz(eps)
    r.set_freeze(2)
    t = 0.0
    tp = np.array(tape, copy=True)
    for s in range(tp.shape[0]):
        r.step(0.0, 1.0, t, 1e300, dt, tp[s])
        t += dt
    return r.get_q()


def gen_adjoint():
    from awcm import gradient as G
    c = ADJ_CASE
    nl, nxc = c["num_levels"], c["nx_coarse"]
    r = oracle.Oracle2D(nl, nxc, nxc, 0.0, 10.0, 0.0, 10.0, bc_kind=2, kind="reference")
    q0 = G.vortex_bumps(r)
    target = G.target_density(r)
    dt = G.stable_dt(q0, 10.0 / (r.nx - 1))
    r.set_q(q0)
    r.prepare(c["tol"])
    qp, masks, levels = r.get_q(), r.get_masks(), r.get_levels()
    # recording run (LF speeds computed), then central differences with the speeds replayed
    r.set_wenoz(c["eps"])
    r.set_freeze(1)
    tape = np.zeros((c["steps"], 3 * (r.nx + r.ny)))
    t = 0.0
    for s in range(c["steps"]):
        r.step(0.0, 1.0, t, 1e300, dt, tape[s])
        t += dt
    q_end = r.get_q()
    dirs = G.unit_directions(qp.shape, c["n_dirs"], c["dir_seed"])
    fd = []
    for d in dirs:
        a = frozen_replay("reference", qp + c["h"] * d, masks, levels, tape, dt, c["eps"], nl, nxc)
        b = frozen_replay("reference", qp - c["h"] * d, masks, levels, tape, dt, c["eps"], nl, nxc)
        fd.append(G.loss_difference(a, b, target, G.active_points(masks)) / (2 * c["h"]))
    return {"adjoint_vortex65": dict(q=qp, masks=masks, levels=levels, tape=tape, target=target, q_end=q_end,
                                     fd=np.array(fd), dt=dt,
                                     params=np.array([nl, nxc, c["tol"], c["eps"], c["steps"], c["n_dirs"],
                                                      c["dir_seed"], c["h"]]))}


def main():
    if not oracle.reference_available():
        oracle.build(with_reference=True)
    groups = {"1d": gen_1d, "2d": gen_2d, "adjoint": gen_adjoint}
    chosen = sys.argv[1:] or list(groups)
    recs = {}
    for g in chosen:
        recs.update(groups[g]())
    for name, rec in recs.items():
        path = os.path.join(HERE, f"{name}.npz")
        np.savez_compressed(path, **rec)
        print(path, os.path.getsize(path))


if __name__ == "__main__":
    main()
