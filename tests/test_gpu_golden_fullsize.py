"""CUDA path against the reference's own outputs (golden fixtures) and at the benchmark sizes.

* golden: tests/golden/*.npz were produced by the reference's code; the GPU must reproduce them.
* full size: the 2049^2 four-quadrant and 4097x1025 double-Mach configurations, first steps,
  bit for bit against the CPU oracle, plus size-independent invariants after more steps
  (nested masks, residue removal, positivity on the active set).
"""
import os

import numpy as np
import pytest

from oracle import Oracle2D

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def corner_free(q):
    keep = np.ones(q.shape[:2], bool)
    keep[:3, :3] = keep[:3, -3:] = keep[-3:, :3] = keep[-3:, -3:] = False
    return q[keep]


@pytest.mark.parametrize("name", ["quad65", "quad129_refsplit", "dmach129x33", "vortex65"])
def test_2d_golden(name, awcm_lib):
    g = dict(np.load(os.path.join(GOLDEN, name + ".npz")))
    nl, nxc, nyc, x0, x1, y0, y1, bc, prob, a, b, tol, cfl, steps = g["params"]
    s = awcm_lib.AWCM2D(int(nl), int(nxc), int(nyc), x0, x1, y0, y1, int(bc))
    s.init_problem(int(prob), a, b)
    assert np.array_equal(s.get_q(), g["q0"])
    t = 0.0
    for k in range(int(steps)):
        out = s.step(tol, cfl, t, 10.0)
        assert out[0] == g["steps"][k][0] and np.array_equal(out[2:6], g["steps"][k][2:6]), k
        t += out[0]
    assert np.array_equal(corner_free(s.get_q()), corner_free(g["q"]))
    assert np.array_equal(s.get_masks(), g["masks"])
    assert np.array_equal(s.get_levels()[:3], g["levels"])


@pytest.mark.parametrize("name", ["sod1d_wenoz_full", "tube0_L5", "tube1_L6", "tube2_L8"])
def test_1d_golden(name, awcm_lib):
    g = dict(np.load(os.path.join(GOLDEN, name + ".npz")))
    if name.startswith("sod"):
        n = 1025
        s = awcm_lib.AWCM1D(7, 17, 0.5 / n, 1 - 0.5 / n)
        s.init_riemann(0.5, (1.0, 0.0, 1.0), (0.125, 0.0, 0.1))
        t_end = 0.2
    else:
        L, nxc, x0, x1 = g["geom"]
        r = g["riemann"]
        s = awcm_lib.AWCM1D(int(L), int(nxc), x0, x1)
        s.init_riemann(r[0], tuple(r[1:4]), tuple(r[4:7]))
        t_end = 0.02
    n, t, upd = s.run(1e-4, 0.5, t_end)
    assert np.array_equal(np.array([n, t, upd]), g["run"])
    assert np.array_equal(s.get_q(), g["q"])
    assert np.array_equal(s.get_masks(), g["masks"])


FULL = {
    "quadrants_2049": (7, 33, 33, (0.0, 1.0, 0.0, 1.0), 0, 0, 0.5, 0.5, 1e-3, 0.4),
    "double_mach_4097x1025": (7, 65, 17, (0.0, 4.0, 0.0, 1.0), 1, 1, 1.4, 0.0, 1e-3, 0.5),
}


@pytest.mark.parametrize("case", list(FULL))
def test_fullsize_first_steps_bit_exact(case, awcm_lib):
    nl, nxc, nyc, dom, bc, prob, a, b, tol, cfl = FULL[case]
    ref = Oracle2D(nl, nxc, nyc, *dom, bc_kind=bc, kind="port")
    gpu = awcm_lib.AWCM2D(nl, nxc, nyc, *dom, bc)
    ref.init_problem(prob, a, b)
    gpu.init_problem(prob, a, b)
    from near_threshold import near_threshold

    t = 0.0
    for k in range(2):
        n_k, e_k = near_threshold((nl, nxc, nyc, *dom, bc), ref.get_q(), ref.get_masks(), tol)
        print(f"{case} step {k}: {n_k} of {e_k} active details within 1e-12 relative of the threshold")
        o_r = ref.step(tol, cfl, t, 10.0)
        o_g = gpu.step(tol, cfl, t, 10.0)
        assert o_g[0] == o_r[0] and np.array_equal(o_g[2:6], o_r[2:6]), (k, o_g, o_r)
        t += o_r[0]
    assert np.array_equal(gpu.get_masks(), ref.get_masks())
    assert np.array_equal(gpu.get_levels()[:3], ref.get_levels()[:3])
    qg, qr = gpu.get_q(), ref.get_q()
    assert np.array_equal(corner_free(qg), corner_free(qr)), float(np.abs(corner_free(qg) - corner_free(qr)).max())


def test_fullsize_invariants(awcm_lib):
    nl, nxc, nyc, dom, bc, prob, a, b, tol, cfl = FULL["quadrants_2049"]
    s = awcm_lib.AWCM2D(nl, nxc, nyc, *dom, bc)
    s.init_problem(prob, a, b)
    t, n, upd, _ = s.advance(tol, cfl, 0.0, 0.3, 40)
    assert n == 40 and upd > 0
    m = s.get_masks()[1:].astype(bool)  # mask0..mask3
    for k in range(3):
        assert not np.any(m[k] & ~m[k + 1]), f"mask{k} not inside mask{k + 1}"
    q = s.get_q()
    inner = q[4:-4, 4:-4]
    off = ~m[0][4:-4, 4:-4]
    assert np.all(inner[off] == 0.0), "residue outside mask0"
    on = m[0][3:-3, 3:-3]
    rho = q[3:-3, 3:-3, 0][on]
    assert np.all(np.isfinite(q)) and np.all(rho > 0)


def test_persistent_prepare_matches_per_phase(awcm_lib):
    """The cooperative persistent PrepareEuler kernel and the per-pass launches agree bit for bit."""
    res = []
    for mode in (1, 0):
        s = awcm_lib.AWCM2D(6, 17, 17, 0.0, 1.0, 0.0, 1.0, 0)
        s.set_prepare_mode(mode)
        s.init_problem(0, 0.5, 0.5)
        s.advance(1e-3, 0.4, 0.0, 0.3, 4)
        res.append((s.get_q(), s.get_masks(), s.get_levels()))
    for x, y in zip(*res):
        assert np.array_equal(x, y)
