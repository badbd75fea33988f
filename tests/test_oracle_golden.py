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
