"""The CPU restatement (oracle port) replays the reference's own outputs bit for bit.

tests/golden/*.npz come from the reference's code compiled from the reference tree
(tests/golden/make_golden.py); the restatement must reproduce every field, mask and level.
"""
import glob
import os

import numpy as np
import pytest

from oracle import Oracle1D, Oracle2D

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
N_SOD = 1025
SOD = dict(num_levels=7, nx_coarse=17, x_min=0.5 / N_SOD, x_max=1 - 0.5 / N_SOD)


def load(name):
    return dict(np.load(os.path.join(GOLDEN, name + ".npz")))


def test_fixtures_present():
    names = {os.path.basename(p)[:-4] for p in glob.glob(os.path.join(GOLDEN, "*.npz"))}
    assert {"sod1d_wenoz_10", "sod1d_weno5_10", "sod1d_wenoz_full", "quad65", "dmach129x33", "vortex65"} <= names


@pytest.mark.parametrize("name", ["sod1d_wenoz_10", "sod1d_weno5_10"])
def test_sod_first_steps(name):
    g = load(name)
    o = Oracle1D(**SOD, scheme=int(g["scheme"]), kind="port")
    o.init_riemann(0.5, (1.0, 0.0, 1.0), (0.125, 0.0, 0.1))
    t = 0.0
    for k, ref in enumerate(g["steps"]):
        out = o.step(1e-4, 0.5, t, 0.2)
        assert np.array_equal(out, ref), (k, out, ref)
        t += out[0]
    assert np.array_equal(o.get_q(), g["q"])
    assert np.array_equal(o.get_masks(), g["masks"])
    assert np.array_equal(o.get_levels(), g["levels"])


def test_sod_full_run():
    g = load("sod1d_wenoz_full")
    o = Oracle1D(**SOD, kind="port")
    o.init_riemann(0.5, (1.0, 0.0, 1.0), (0.125, 0.0, 0.1))
    n, t, upd = o.run(1e-4, 0.5, 0.2)
    assert np.array_equal(np.array([n, t, upd]), g["run"])
    assert (n, upd) == (897, 151533.0)
    assert np.array_equal(o.get_q(), g["q"])
    assert np.array_equal(o.get_masks(), g["masks"])


@pytest.mark.parametrize("name", ["tube0_L5", "tube1_L6", "tube2_L8"])
def test_uneven_tubes(name):
    g = load(name)
    L, nxc, x0, x1 = g["geom"]
    r = g["riemann"]
    o = Oracle1D(int(L), int(nxc), x0, x1, kind="port")
    o.init_riemann(r[0], tuple(r[1:4]), tuple(r[4:7]))
    n, t, upd = o.run(1e-4, 0.5, 0.02)
    assert np.array_equal(np.array([n, t, upd]), g["run"])
    assert np.array_equal(o.get_q(), g["q"])
    assert np.array_equal(o.get_masks(), g["masks"])


@pytest.mark.parametrize("name", ["quad65", "quad129_refsplit", "dmach129x33", "vortex65"])
def test_2d_steps(name):
    g = load(name)
    nl, nxc, nyc, x0, x1, y0, y1, bc, prob, a, b, tol, cfl, steps = g["params"]
    o = Oracle2D(int(nl), int(nxc), int(nyc), x0, x1, y0, y1, bc_kind=int(bc), kind="port")
    o.init_problem(int(prob), a, b)
    assert np.array_equal(o.get_q(), g["q0"])
    t = 0.0
    for k in range(int(steps)):
        out = o.step(tol, cfl, t, 10.0)
        assert np.array_equal(out, g["steps"][k]), (k, out, g["steps"][k])
        t += out[0]
    q = o.get_q()
    keep = np.ones(q.shape[:2], bool)
    keep[:3, :3] = keep[:3, -3:] = keep[-3:, :3] = keep[-3:, -3:] = False
    assert np.array_equal(q[keep], g["q"][keep])
    assert np.array_equal(o.get_masks(), g["masks"])
    assert np.array_equal(o.get_levels()[:3], g["levels"])


def test_frozen_gradient_fixture():
    """Frozen-mask mode with the LF speeds replayed and WENO-Z eps 1e-6: the restatement gives the
    reference's end state and its central differences of the loss on all 16 directions, bit for bit."""
    from awcm import gradient as G

    g = load("adjoint_vortex65")
    nl, nxc, tol, eps, steps, n_dirs, seed, h = g["params"]
    nl, nxc, steps, n_dirs, seed = int(nl), int(nxc), int(steps), int(n_dirs), int(seed)
    dt = float(g["dt"])

    def replay(q):
        o = Oracle2D(nl, nxc, nxc, 0.0, 10.0, 0.0, 10.0, bc_kind=2, kind="port")
        o.set_q(q)
        o.set_masks(g["masks"])
        o.set_levels(g["levels"])
        o.set_wenoz(eps)
        o.set_freeze(2)
        t, tape = 0.0, np.array(g["tape"], copy=True)
        for s in range(steps):
            o.step(0.0, 1.0, t, 1e300, dt, tape[s])
            t += dt
        return o.get_q()

    assert np.array_equal(replay(g["q"]), g["q_end"])
    dirs = G.unit_directions(g["q"].shape, n_dirs, seed)
    for k in (0, 5, 11):
        a, b = replay(g["q"] + h * dirs[k]), replay(g["q"] - h * dirs[k])
        assert G.loss_difference(a, b, g["target"], G.active_points(g["masks"])) / (2 * h) == g["fd"][k]


def test_frozen_gradient_workload_builder():
    """The workload builder reproduces the fixture's target and prepared state from the seeds."""
    from awcm import gradient as G

    g = load("adjoint_vortex65")
    nl, nxc, tol = int(g["params"][0]), int(g["params"][1]), float(g["params"][2])
    o = Oracle2D(nl, nxc, nxc, 0.0, 10.0, 0.0, 10.0, bc_kind=2, kind="port")
    q0 = G.vortex_bumps(o)
    assert np.array_equal(G.target_density(o), g["target"])
    assert G.stable_dt(q0, 10.0 / (o.nx - 1)) == float(g["dt"])
    o.set_q(q0)
    o.prepare(tol)
    assert np.array_equal(o.get_q(), g["q"])
    assert np.array_equal(o.get_masks(), g["masks"])


def test_near_threshold_report():
    """The near-threshold counter finds a detail placed exactly on the threshold and none on a
    state whose details are far from it."""
    from near_threshold import detail_ratios, near_threshold

    g = load("quad65")
    nl, nxc, nyc, x0, x1, y0, y1, bc = g["params"][:8]
    geom = (int(nl), int(nxc), int(nyc), x0, x1, y0, y1, int(bc))
    o = Oracle2D(*geom[:7], bc_kind=geom[7], kind="port")
    o.set_q(g["q0"])
    masks = o.get_masks()
    r = detail_ratios(geom, g["q0"], masks, 1.0)
    nz = r[r > 0]
    assert nz.size > 0
    tol = float(nz[0])  # a threshold equal to one detail's magnitude
    n, examined = near_threshold(geom, g["q0"], masks, tol)
    assert n >= 1 and examined == r.size
    n2, _ = near_threshold(geom, g["q0"], masks, tol * 1.5)
    assert n2 <= n
