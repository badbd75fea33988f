"""2D parity: the CUDA path against the CPU oracle (restatement of the reference), bit for bit.

Masks and levels must be identical; conserved fields are compared exactly as well (the kernels
keep the reference's operation order under --fmad=false), with the 1e-11 relative L-infinity
bound of the path's contract checked separately so a failure says which bar was missed.
Corner ghost cells are excluded: no boundary manager of the reference fills them and no stencil
reads them.
"""
import numpy as np
import pytest

import oracle
from oracle import Oracle2D

pytestmark = pytest.mark.gpu

REL_TOL = 1e-11

CASES = {
    # name: (num_levels, nx_coarse, ny_coarse, domain, bc, problem, a, b, tol, cfl)
    "quad65": (4, 9, 9, (0.0, 1.0, 0.0, 1.0), 0, 0, 0.5, 0.5, 1e-3, 0.4),
    "quad129": (5, 9, 9, (0.0, 1.0, 0.0, 1.0), 0, 0, 0.5, 0.5, 1e-3, 0.4),
    "quad_ref_split": (5, 9, 9, (0.0, 1.0, 0.0, 1.0), 0, 0, 0.8, 0.8, 1e-4, 0.5),
    "dmach": (4, 17, 5, (0.0, 4.0, 0.0, 1.0), 1, 1, 1.4, 0.0, 1e-3, 0.5),
    "vortex": (4, 9, 9, (0.0, 10.0, 0.0, 10.0), 2, 2, 5.0, 5.0, 1e-3, 0.4),
    "shock_vortex": (5, 9, 9, (-16.0, 8.0, -12.0, 12.0), 3, 3, 2.0, 0.0, 1e-3, 0.4),
}


def corner_free(q):
    keep = np.ones(q.shape[:2], bool)
    keep[:3, :3] = keep[:3, -3:] = keep[-3:, :3] = keep[-3:, -3:] = False
    return q[keep]


def rel_linf(a, b):
    scale = max(np.abs(b).max(), 1e-300)
    return np.abs(a - b).max() / scale


def make(case, awcm):
    nl, nxc, nyc, dom, bc, prob, a, b, tol, cfl = CASES[case]
    ref = Oracle2D(nl, nxc, nyc, *dom, bc_kind=bc, kind="port")
    gpu = awcm.AWCM2D(nl, nxc, nyc, *dom, bc_kind=bc)
    ref.init_problem(prob, a, b)
    gpu.init_problem(prob, a, b)
    return ref, gpu, tol, cfl


def assert_same_state(gpu, ref, what, levels=(0, 1, 2)):
    qg, qr = gpu.get_q(), ref.get_q()
    assert rel_linf(corner_free(qg), corner_free(qr)) <= REL_TOL, f"{what}: field beyond 1e-11"
    assert np.array_equal(corner_free(qg), corner_free(qr)), f"{what}: field not bit-identical"
    mg, mr = gpu.get_masks(), ref.get_masks()
    assert np.array_equal(mg, mr), f"{what}: masks differ at {np.argwhere(mg != mr)[:5]}"
    lg, lr = gpu.get_levels(), ref.get_levels()
    for l in levels:
        assert np.array_equal(lg[l], lr[l]), f"{what}: level{l} differs at {np.argwhere(lg[l] != lr[l])[:5]}"


@pytest.mark.parametrize("case", list(CASES))
def test_initial_state_identical(case, awcm_lib):
    ref, gpu, _, _ = make(case, awcm_lib)
    assert np.array_equal(gpu.get_q(), ref.get_q())
    assert np.array_equal(gpu.get_masks(), ref.get_masks())


@pytest.mark.parametrize("case", ["quad65", "dmach", "vortex"])
def test_forward_transform(case, awcm_lib):
    ref, gpu, tol, _ = make(case, awcm_lib)
    ref.fwt(tol)
    gpu.fwt(tol)
    assert np.array_equal(gpu.get_q()[..., 0], ref.get_q()[..., 0])
    assert np.array_equal(gpu.get_masks()[1], ref.get_masks()[1])


@pytest.mark.parametrize("case", ["quad65", "quad129", "dmach", "vortex"])
def test_prepare(case, awcm_lib):
    ref, gpu, tol, _ = make(case, awcm_lib)
    for _ in range(2):
        ref.prepare(tol)
        gpu.prepare(tol)
        assert_same_state(gpu, ref, f"{case} prepare")


def test_manager_passes_in_sequence(awcm_lib):
    """The AWCM_MANAGER_2D passes one by one, in PrepareEuler's order, each checked on its own."""
    ref, gpu, tol, _ = make("quad129", awcm_lib)
    ref.fwt(tol)
    gpu.fwt(tol)
    seq = [(oracle.BAND, 0, 0), (oracle.AAZ, 0, 0), (oracle.CR, 0, 0), (oracle.CL, 0, 0),
           (oracle.APD, 0, 0), (oracle.CR, 0, 0), (oracle.CL, 0, 1), (oracle.AAZ, 0, 0), (oracle.CR, 0, 0),
           (oracle.RR, 0, 0)]
    for op, mask_id, level_id in seq:
        ref.manager(op, mask_id, level_id)
        gpu.manager(op, mask_id, level_id)
        what = f"op {op}"
        assert np.array_equal(gpu.get_masks(), ref.get_masks()), what
        assert np.array_equal(gpu.get_levels()[:2], ref.get_levels()[:2]), what
        assert np.array_equal(corner_free(gpu.get_q()), corner_free(ref.get_q())), what
    ref.iwt(0)
    gpu.iwt(0)
    ref.interpolate(4, 0)
    gpu.interpolate(4, 0)
    assert np.array_equal(corner_free(gpu.get_q()), corner_free(ref.get_q()))


@pytest.mark.parametrize("case", list(CASES))
def test_steps(case, awcm_lib):
    from near_threshold import near_threshold

    ref, gpu, tol, cfl = make(case, awcm_lib)
    nl, nxc, nyc, dom, bc = CASES[case][:5]
    t, t_end = 0.0, 10.0
    near, examined = 0, 0
    for k in range(6):
        n_k, e_k = near_threshold((nl, nxc, nyc, *dom, bc), ref.get_q(), ref.get_masks(), tol)
        near, examined = near + n_k, examined + e_k
        o_r = ref.step(tol, cfl, t, t_end)
        o_g = gpu.step(tol, cfl, t, t_end)
        assert o_g[0] == o_r[0], f"step {k}: dt {o_g[0]!r} vs {o_r[0]!r}"
        assert np.array_equal(o_g[2:6], o_r[2:6]), f"step {k}: mask sizes"
        assert_same_state(gpu, ref, f"{case} step {k}")
        t += o_r[0]
    # masks are compared bit for bit above, near-threshold points included; the count is reported
    print(f"{case}: {near} of {examined} active details within 1e-12 relative of the threshold")


def test_output_time_clipping(awcm_lib):
    ref, gpu, tol, cfl = make("quad65", awcm_lib)
    o_r = ref.step(tol, cfl, 0.0, 1e-4)
    o_g = gpu.step(tol, cfl, 0.0, 1e-4)
    assert o_r[1] == 1 and o_g[1] == 1 and o_g[0] == o_r[0] == 1e-4
    assert_same_state(gpu, ref, "clipped step")


def test_advance_matches_steps(awcm_lib):
    """Graph-replayed steps (device-held t) give the same state as host-driven steps."""
    ref, gpu, tol, cfl = make("quad65", awcm_lib)
    t = 0.0
    for _ in range(5):
        t += ref.step(tol, cfl, t, 0.05)[0]
    tg, n, upd, _ = gpu.advance(tol, cfl, 0.0, 0.05, 5)
    assert n == 5 and tg == t
    assert_same_state(gpu, ref, "advance")


def test_run_to_end(awcm_lib):
    ref, gpu, tol, cfl = make("quad65", awcm_lib)
    n_r, t_r, u_r = ref.run(tol, cfl, 0.02)
    n_g, t_g, u_g = gpu.run(tol, cfl, 0.02)
    assert (n_g, t_g, u_g) == (n_r, t_r, u_r)
    assert_same_state(gpu, ref, "run")
