"""Parity where the benchmarks run: developed flow at full size, a whole run, the batched sizes.

* Developed flow, full size: the GPU runs the 2049^2 four-quadrant problem 1500 steps (the
  shocks interacting, the active set several times its initial size) and the 4097x1025 double
  Mach problem 800 steps, saves its state to the binary state file, and both the GPU and the
  CPU oracle load that file and take three steps in lockstep: dt, mask sizes, masks, levels and
  fields bit for bit.
* Whole run: the 513^2 four-quadrant problem from its initial state to t_end = 0.3 on both
  sides: step count, final time, sum of |mask0| over the steps and the final state.
* Batched sizes: eight tubes of the seeded 512-tube workload (three with Jmax 13, the largest
  and shared-memory-heaviest instances, and one of each Jmax 8..12) advanced as one batch to
  t_end = 0.15 against the oracle run instance by instance.
The oracle runs in a process pool started with `spawn` (a pool forked after CUDA is initialised
can hang).
"""
import concurrent.futures as cf
import multiprocessing as mp

import numpy as np
import pytest

import oracle
from oracle import Oracle2D
from oracle.state_format import read_state

pytestmark = pytest.mark.gpu


def corner_free(q):
    keep = np.ones(q.shape[:2], bool)
    keep[:3, :3] = keep[:3, -3:] = keep[-3:, :3] = keep[-3:, -3:] = False
    return q[keep]


DEVELOPED = {
    # name: (num_levels, nx_coarse, ny_coarse, domain, bc, problem, a, b, tol, cfl, t_end, steps)
    "quadrants_2049_step1500": (7, 33, 33, (0.0, 1.0, 0.0, 1.0), 0, 0, 0.5, 0.5, 1e-3, 0.4, 0.3, 1500),
    "double_mach_4097x1025_step800": (7, 65, 17, (0.0, 4.0, 0.0, 1.0), 1, 1, 1.4, 0.0, 1e-3, 0.5, 0.2, 800),
}


@pytest.mark.parametrize("case", list(DEVELOPED))
def test_developed_flow_lockstep_from_state_file(tmp_path, awcm_lib, case):
    from near_threshold import near_threshold

    nl, nxc, nyc, dom, bc, prob, a, b, tol, cfl, t_end, steps = DEVELOPED[case]
    gpu = awcm_lib.AWCM2D(nl, nxc, nyc, *dom, bc)
    gpu.init_problem(prob, a, b)
    t, n, _, _ = gpu.advance(tol, cfl, 0.0, t_end, steps)
    assert n == steps
    p = tmp_path / "developed.bin"
    gpu.save_state(p, t, steps)
    r = read_state(p)
    ref = Oracle2D(nl, nxc, nyc, *dom, bc_kind=bc, kind="port")
    ref.set_q(r["q"])
    ref.set_masks(r["masks"])
    ref.set_levels(r["levels"])
    t2, _ = gpu.load_state(p)
    assert t2 == r["t"] == t
    print(f"{case}: t = {t:.6g} after {steps} steps, |mask3| = {int(r['masks'][4].sum())}")
    near, examined = 0, 0
    for k in range(3):
        n_k, e_k = near_threshold((nl, nxc, nyc, *dom, bc), ref.get_q(), ref.get_masks(), tol)
        near, examined = near + n_k, examined + e_k
        o_r = ref.step(tol, cfl, t, t_end)
        o_g = gpu.step(tol, cfl, t, t_end)
        assert o_g[0] == o_r[0], f"step {k}: dt {o_g[0]!r} vs {o_r[0]!r}"
        assert np.array_equal(o_g[2:6], o_r[2:6]), f"step {k}: mask sizes {o_g[2:6]} vs {o_r[2:6]}"
        t += o_r[0]
        mg, mr = gpu.get_masks(), ref.get_masks()
        assert np.array_equal(mg, mr), f"step {k}: masks differ at {np.argwhere(mg != mr)[:5]}"
        assert np.array_equal(gpu.get_levels()[:3], ref.get_levels()[:3]), f"step {k}: levels"
        qg, qr = corner_free(gpu.get_q()), corner_free(ref.get_q())
        assert np.abs(qg - qr).max() <= 1e-11 * np.abs(qr).max(), f"step {k}: field beyond 1e-11"
        assert np.array_equal(qg, qr), f"step {k}: field not bit-identical"
    print(f"{case}: {near} of {examined} active details within 1e-12 relative of the threshold")


def test_quadrants_513_whole_run(awcm_lib):
    geom = (6, 17, 17, 0.0, 1.0, 0.0, 1.0)
    gpu = awcm_lib.AWCM2D(*geom, 0)
    ref = Oracle2D(*geom, bc_kind=0, kind="port")
    gpu.init_problem(0, 0.5, 0.5)
    ref.init_problem(0, 0.5, 0.5)
    n_g, t_g, u_g = gpu.run(1e-3, 0.4, 0.3)
    n_r, t_r, u_r = ref.run(1e-3, 0.4, 0.3)
    print(f"513^2 to t = 0.3: {n_r} steps, sum |mask0| = {u_r:.0f}")
    assert (n_g, t_g, u_g) == (n_r, t_r, u_r)
    assert np.array_equal(gpu.get_masks(), ref.get_masks())
    assert np.array_equal(gpu.get_levels()[:3], ref.get_levels()[:3])
    assert np.array_equal(corner_free(gpu.get_q()), corner_free(ref.get_q()))


def batch_sample():
    from awcm import workloads

    tubes = workloads.shock_tubes(512)
    pick = [k for k, t in enumerate(tubes) if t["jmax"] == 13][:3]
    for j in range(8, 13):
        pick.append(next(k for k, t in enumerate(tubes) if t["jmax"] == j))
    return [tubes[k] for k in pick], pick


def test_batched_tubes_to_t_end(awcm_lib):
    from awcm import workloads

    tol, cfl, t_end = 1e-4, 0.5, 0.15
    tubes, pick = batch_sample()
    ctx = mp.get_context("spawn")
    with cf.ProcessPoolExecutor(max_workers=len(tubes), mp_context=ctx) as ex:
        futs = [ex.submit(oracle.run_tube, t, tol, cfl, t_end) for t in tubes]
        b = workloads.make_batch(awcm_lib, tubes)
        b.set_run(tol, cfl, 0.0, t_end)
        for _ in range(400):
            b.steps(250)
            if b.totals()[2] == b.n:
                break
        res = [f.result() for f in futs]
    for k, (t, (n, tt, upd, q, m, lv)) in enumerate(zip(tubes, res)):
        s = b.status(k)
        what = f"tube {pick[k]} (Jmax {t['jmax']})"
        print(f"{what}: {n} steps, sum |mask0| = {upd:.0f}")
        assert s[3] == 1 and s[14] == 0, f"{what}: status {s}"
        assert (int(s[4]), s[0], s[13]) == (n, tt, upd), f"{what}: {s[[4, 0, 13]]} vs {(n, tt, upd)}"
        assert np.array_equal(b.get_q(k), q), f"{what}: field"
        assert np.array_equal(b.get_masks(k), m), f"{what}: masks"
        assert np.array_equal(b.get_levels(k), lv), f"{what}: levels"
