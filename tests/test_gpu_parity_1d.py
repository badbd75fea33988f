"""1D parity: the CUDA path (single instances and batches) against the CPU oracle, bit for bit."""
import numpy as np
import pytest

import oracle
from oracle import Oracle1D

pytestmark = pytest.mark.gpu

N_SOD = 1025
DXF = 1.0 / N_SOD
SOD = dict(num_levels=7, nx_coarse=17, x_min=0.5 * DXF, x_max=1 - 0.5 * DXF)
LEFT, RIGHT = (1.0, 0.0, 1.0), (0.125, 0.0, 0.1)


def make(awcm, scheme=0, **kw):
    geo = dict(SOD, **kw)
    ref = Oracle1D(geo["num_levels"], geo["nx_coarse"], geo["x_min"], geo["x_max"], scheme=scheme, kind="port")
    gpu = awcm.AWCM1D(geo["num_levels"], geo["nx_coarse"], geo["x_min"], geo["x_max"], scheme=scheme)
    ref.init_riemann(0.5, LEFT, RIGHT)
    gpu.init_riemann(0.5, LEFT, RIGHT)
    return ref, gpu


def assert_same(gpu, ref, what):
    assert np.array_equal(gpu.get_q(), ref.get_q()), f"{what}: field"
    assert np.array_equal(gpu.get_masks(), ref.get_masks()), f"{what}: masks"
    assert np.array_equal(gpu.get_levels(), ref.get_levels()), f"{what}: levels"


def test_initial_state(awcm_lib):
    ref, gpu = make(awcm_lib)
    assert_same(gpu, ref, "init")


def test_prepare(awcm_lib):
    ref, gpu = make(awcm_lib)
    ref.prepare(1e-4)
    gpu.prepare(1e-4)
    assert_same(gpu, ref, "prepare")


def test_manager_passes_in_sequence(awcm_lib):
    """The AWCM_MANAGER_1D passes one by one, in PrepareEuler's order, each checked on its own."""
    ref, gpu = make(awcm_lib)
    ref.fwt(1e-4)
    gpu.fwt(1e-4)
    seq = [(oracle.BAND, 0, 0), (oracle.AAZ, 0, 0), (oracle.CR, 0, 0), (oracle.CL, 0, 0),
           (oracle.APD, 0, 0), (oracle.CR, 0, 0), (oracle.CL, 0, 1), (oracle.RR, 0, 0)]
    for op, mask_id, level_id in seq:
        ref.manager(op, mask_id, level_id)
        gpu.manager(op, mask_id, level_id)
        assert_same(gpu, ref, f"op {op}")
    ref.iwt(0)
    gpu.iwt(0)
    assert_same(gpu, ref, "iwt")


def test_interpolate_and_boundary_fill(awcm_lib):
    """The typed single passes WAVELET_1D::InterpolateEuler(mask_temp -> mask3) and the
    transmissive ghost fill, on a stepped state with a perturbed field."""
    ref, gpu = make(awcm_lib)
    t = 0.0
    for _ in range(40):
        o_r = ref.step(1e-4, 0.5, t, 0.2)
        gpu.step(1e-4, 0.5, t, 0.2)
        t += o_r[0]
    assert_same(gpu, ref, "40 steps")
    q = ref.get_q() + np.random.default_rng(3).uniform(0, 1e-3, ref.get_q().shape)
    for o in (ref, gpu):
        o.set_q(q)
        o.interpolate(4, 3)
    assert_same(gpu, ref, "interpolate")
    for o in (ref, gpu):
        o.apply_bc()
    assert_same(gpu, ref, "boundary fill")
    for o in (ref, gpu):
        o.iwt(3)
    assert_same(gpu, ref, "inverse transform")


@pytest.mark.parametrize("scheme", [0, 1])
def test_steps(scheme, awcm_lib):
    ref, gpu = make(awcm_lib, scheme=scheme)
    t = 0.0
    for k in range(25):
        o_r = ref.step(1e-4, 0.5, t, 0.2)
        o_g = gpu.step(1e-4, 0.5, t, 0.2)
        assert np.array_equal(o_g, o_r), f"step {k}: {o_g} vs {o_r}"
        assert_same(gpu, ref, f"scheme {scheme} step {k}")
        t += o_r[0]


def test_sod_full_run(awcm_lib):
    """The 1D Sod benchmark case to t = 0.2: same step count, same updates, same final state."""
    ref, gpu = make(awcm_lib)
    n_r, t_r, u_r = ref.run(1e-4, 0.5, 0.2)
    n_g, t_g, u_g = gpu.run(1e-4, 0.5, 0.2)
    assert (n_g, t_g, u_g) == (n_r, t_r, u_r) == (897, 0.2, 151533.0)
    assert_same(gpu, ref, "final")


def test_batch_uneven_matches_single(awcm_lib):
    """Uneven instances advanced in one launch equal the oracle run instance by instance."""
    rng = np.random.default_rng(7)
    levels = [5, 7, 6, 8, 5, 9]
    tubes = []
    for L in levels:
        nx = 16 * 2 ** (L - 1) + 1
        dxf = 1.0 / nx
        tubes.append((L, 0.5 * dxf, 1 - 0.5 * dxf, rng.uniform(0.3, 0.7),
                       (10 ** rng.uniform(-1, 1), rng.uniform(-1, 1), 10 ** rng.uniform(-1, 1)),
                       (10 ** rng.uniform(-1, 1), rng.uniform(-1, 1), 10 ** rng.uniform(-1, 1))))
    b = awcm_lib.AWCM1DBatch([t[0] for t in tubes], 17, [t[1] for t in tubes], [t[2] for t in tubes])
    refs = []
    for k, (L, x0, x1, xi, l, r) in enumerate(tubes):
        b.init_riemann(k, xi, l, r)
        o = Oracle1D(L, 17, x0, x1, kind="port")
        o.init_riemann(xi, l, r)
        refs.append(o)
    t_end = 0.01
    b.set_run(1e-4, 0.5, 0.0, t_end)
    for _ in range(40):
        b.steps(100)
        if b.totals()[2] == b.n:
            break
    for k, o in enumerate(refs):
        n, t, upd = o.run(1e-4, 0.5, t_end)
        s = b.status(k)
        assert s[3] == 1 and int(s[4]) == n and s[0] == t and s[13] == upd, (k, s[:5], n, t)
        assert np.array_equal(b.get_q(k), o.get_q()), f"instance {k}"
        assert np.array_equal(b.get_masks(k), o.get_masks()), f"instance {k} masks"


@pytest.mark.parametrize("threads,ctas", [(64, 0), (128, 2), (256, 0), (512, 0), (768, 0)])
def test_launch_shapes_agree(threads, ctas, awcm_lib):
    """Every launch shape the autotuner may pick gives the oracle's run, bit for bit (the step's
    reductions are order-free and its worklists keep the point order)."""
    ref, gpu = make(awcm_lib)
    gpu.b.set_launch(threads, ctas)
    n_r, t_r, u_r = ref.run(1e-4, 0.5, 0.05)
    n_g, t_g, u_g = gpu.run(1e-4, 0.5, 0.05)
    assert (n_g, t_g, u_g) == (n_r, t_r, u_r)
    assert_same(gpu, ref, f"{threads}x{ctas}")


def _uneven_batch(awcm_lib, seed=7):
    rng = np.random.default_rng(seed)
    tubes = []
    for L in [5, 7, 6, 8, 5, 9]:
        nx = 16 * 2 ** (L - 1) + 1
        dxf = 1.0 / nx
        tubes.append((L, 0.5 * dxf, 1 - 0.5 * dxf, rng.uniform(0.3, 0.7),
                       (10 ** rng.uniform(-1, 1), rng.uniform(-1, 1), 10 ** rng.uniform(-1, 1)),
                       (10 ** rng.uniform(-1, 1), rng.uniform(-1, 1), 10 ** rng.uniform(-1, 1))))
    b = awcm_lib.AWCM1DBatch([t[0] for t in tubes], 17, [t[1] for t in tubes], [t[2] for t in tubes])
    refs = []
    for k, (L, x0, x1, xi, l, r) in enumerate(tubes):
        b.init_riemann(k, xi, l, r)
        o = Oracle1D(L, 17, x0, x1, kind="port")
        o.init_riemann(xi, l, r)
        refs.append(o)
    return b, refs


@pytest.mark.parametrize("max_steps", [None, 7])
def test_batch_run_to_end(max_steps, awcm_lib):
    """awcm1d_batch_run: every instance run to t_end (or max_steps steps) in one launch, each on its
    CTA back to back, equals the oracle run instance by instance."""
    b, refs = _uneven_batch(awcm_lib)
    t_end = 0.01
    b.set_run(1e-4, 0.5, 0.0, t_end)
    if max_steps is None:
        b.run_all()
    else:
        b.run_all(max_steps)
    b.sync()
    for k, o in enumerate(refs):
        n, t, upd = o.run(1e-4, 0.5, t_end, (1 << 30) if max_steps is None else max_steps)
        s = b.status(k)
        assert int(s[4]) == n and s[0] == t and s[13] == upd, (k, s[:5], n, t)
        if max_steps is None:
            assert s[3] == 1, (k, s[:5])
        assert np.array_equal(b.get_q(k), o.get_q()), f"instance {k}"
        assert np.array_equal(b.get_masks(k), o.get_masks()), f"instance {k} masks"
        assert np.array_equal(b.get_levels(k), o.get_levels()), f"instance {k} levels"
