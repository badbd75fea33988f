#!/usr/bin/env python
"""Benchmark of the B200 AWCM compressible-Euler path.

Headline workload: the 2D four-quadrant Riemann problem on [0,1]^2 split at (0.5, 0.5), 2049^2
finest nodes (nx_coarse 33, 7 levels: Jmin 5 .. Jmax 11), threshold 1e-3, CFL 0.4, WENO-Z + Roe,
SSP-RK3, transmissive boundaries, FP64.  One step = one full AWCM RK3 step (PrepareEuler, CFL,
three stages, PostProcessEuler).  Metric: active-point RK3 updates per second, i.e. the sum over
the timed steps of |mask0| divided by the device time of those steps.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

N > 1 (launched by torch.distributed.run) runs N independent replicas, one per GPU: the path has
no data-parallel split of one instance, and batched instances need no exchange.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "c_pp-library_b200")
for _p in (ROOT, PKG):
    if _p not in sys.path:
        sys.path.insert(0, _p)

WORKLOAD = {
    "workload": "2D four-quadrant Riemann problem, 2049x2049 finest (Jmin 5, Jmax 11), eps 1e-3, "
                "CFL 0.4, WENO-Z+Roe, SSP-RK3, transmissive, t_end 0.3",
    "num_levels": 7, "nx_coarse": 33, "ny_coarse": 33, "domain": [0.0, 1.0, 0.0, 1.0],
    "split": [0.5, 0.5], "tol": 1e-3, "cfl": 0.4, "t_end": 0.3,
}
# The two other AWCM Euler configurations of the benchmark set, reported beside the headline.
DOUBLE_MACH = {
    "workload": "2D Mach-10 double-Mach reflection, 4097x1025 finest (65x17 coarse, 7 levels) on [0,4]x[0,1], "
                "eps 1e-3, CFL 0.5, WENO-Z+Roe, SSP-RK3, reflecting wall for x > 1/6 and exact moving-shock top, "
                "t_end 0.2",
    "num_levels": 7, "nx_coarse": 65, "ny_coarse": 17, "domain": [0.0, 4.0, 0.0, 1.0], "bc": 1, "problem": 1,
    "a": 1.4, "b": 0.0, "tol": 1e-3, "cfl": 0.5, "t_end": 0.2,
}
SOD = {
    "workload": "1D Sod shock tube, 1025 cell-centred nodes on [0,1] (Jmin 4, Jmax 10), interface 0.5, eps 1e-4, "
                "CFL 0.5, WENO-Z+Roe, SSP-RK3, transmissive, t_end 0.2 (one instance, whole run)",
    "num_levels": 7, "nx_coarse": 17, "n": 1025, "tol": 1e-4, "cfl": 0.5, "t_end": 0.2,
}
# Step of the headline run whose state is the late timing window (developed flow: the four
# waves interacting, the active set several times its initial size).
LATE_STEP = 2000
METRIC = "active-pt RK3 updates/s"
UNIT = "updates/s"
# Algorithmic FP64 operations of one 2D WENO-Z/Roe face flux in the reference
# (WENOZ_EULER_SOLVER_2D::ComputeFluxX, WENOZ.h:236-277): 589 add, 643 mul, 113 div, 9 sqrt.
FLOPS_PER_FACE = 1354
L2_BYTES = 126 * 2 ** 20


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=60)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=15.0, help="CPU-baseline sample budget")
    ap.add_argument("--no-batched", action="store_true", help="skip the batched shock-tube comparison")
    ap.add_argument("--no-adjoint", action="store_true", help="skip the adjoint/forward timing")
    ap.add_argument("--no-full-run", action="store_true", help="skip the whole-run and late-window figures")
    ap.add_argument("--no-configs", action="store_true", help="skip the double-Mach and 1D Sod lines")
    ap.add_argument("--capture", type=int, default=-1,
                    help="profiling mode: K graph-replayed steps, then one eagerly launched step; prints its phases")
    ap.add_argument("--capture-batch", type=int, default=-1,
                    help="profiling mode: the 512-tube batch, K graph-replayed RK3 steps (launches 1..K of k_step1d)")
    ap.add_argument("--capture-skip", type=int, default=0,
                    help="with --capture-batch: S steps before the K (k_step1d launches S+1..S+K; at S = 24000 only "
                         "the four slowest Jmax-13 tubes are still running)")
    return ap.parse_args()


def dist_env():
    return int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("LOCAL_RANK", "0"))


# ------------------------------------------------------------------------------------------ clocks
class ClockSampler:
    """nvidia-smi clock/throttle samples every 200 ms while the timed region runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-lms", "200", "-i", str(self.gpu)], stdout=open(self.path, "w"),
                                         stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        rows = []
        try:
            for line in open(self.path):
                parts = [p.strip() for p in line.split(",")]
                if len(parts) >= 9 and parts[1].replace(".", "").isdigit():
                    rows.append(parts)
        except Exception:
            pass
        finally:
            try:
                os.unlink(self.path)
            except Exception:
                pass
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in rows]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            for n, v in zip(names, r[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": float(rows[0][2]), "reasons": sorted(reasons),
                "samples": len(rows), "power_w_max": max(float(r[3]) for r in rows if r[3].replace(".", "").isdigit())}


# ------------------------------------------------------------------------------------- CPU arms
def reference_solver(w=WORKLOAD, state_file=None):
    """The reference's own 2D code (oracle/_ref), all host threads, on workload `w`: from its
    initial state, or from a state file written by the GPU run."""
    import oracle

    if not oracle.reference_available():
        return None, "reference build (oracle/_ref) not present"
    s = oracle.Oracle2D(w["num_levels"], w["nx_coarse"], w["ny_coarse"], *w["domain"], bc_kind=w.get("bc", 0),
                        kind="reference")
    if state_file is None:
        s.init_problem(w.get("problem", 0), *(w["split"] if "split" in w else (w["a"], w["b"])))
    else:
        from oracle.state_format import read_state

        r = read_state(state_file)
        s.set_q(r["q"])
        s.set_masks(r["masks"])
        s.set_levels(r["levels"])
    return s, None


def time_reference(steps_max: int, seconds: float, warmup: int = 0, w=WORKLOAD, state_file=None, t0_run=0.0):
    """Steps warmup+1 .. warmup+steps_max of the reference solver (at most `seconds` of timed
    work); returns (updates/s, steps, wall, threads)."""
    s, why = reference_solver(w, state_file)
    if s is None:
        return None, why
    t = t0_run
    for _ in range(warmup):
        t += s.step(w["tol"], w["cfl"], t, w["t_end"])[0]
    upd, n = 0.0, 0
    t0 = time.perf_counter()
    while n < steps_max:
        o = s.step(w["tol"], w["cfl"], t, w["t_end"])
        t += o[0]
        upd += o[2]
        n += 1
        if time.perf_counter() - t0 > seconds:
            break
    wall = time.perf_counter() - t0
    return {"value": upd / wall, "steps": n, "wall_s": wall, "cores": s.threads, "warmup": warmup}, None


def run_reference_arm(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return
    os.environ.setdefault("OMP_NUM_THREADS", str(os.cpu_count()))
    # the GPU arm's window: warm-up steps 1..W untimed, steps W+1..W+K timed (W >= 3 there too)
    k = max(1, min(args.steps, 400))
    w = max(3, args.warmup)
    r, why = time_reference(k, 1e9, warmup=w)
    if r is None:
        print(json.dumps({"impl": "reference", "unavailable": why}))
        return
    line = {
        "impl": "reference", "metric": METRIC, "value": r["value"], "unit": UNIT, "n_gpus": world,
        "window": {"first_step": w + 1, "last_step": w + r["steps"]},
        "steps": r["steps"], "warmup": w, "ms_per_step": 1e3 * r["wall_s"] / r["steps"], "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (deterministic initial state)",
        "config": {k2: v for k2, v in WORKLOAD.items()},
        "cpu_baseline": {"value": r["value"], "unit": UNIT, "cores": r["cores"], "kind": "reference",
                         "sample": f"steps {w + 1}..{w + r['steps']} of the workload from its initial state "
                                   f"(reference code compiled from the reference tree, OpenMP {r['cores']} threads)"},
        "e2e": {"value": r["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


# ------------------------------------------------------------------------- batched shock tubes
BATCHED = {
    "workload": "512 seeded 1D shock tubes, Jmin 4, Jmax uniform in {8..13} (257..8193 points), eps 1e-4, "
                "CFL 0.5, WENO-Z+Roe, t_end 0.15; rho/p log-uniform [0.1,10], u uniform [-1,1], interface U[0.3,0.7]",
    "instances": 512, "tol": 1e-4, "cfl": 0.5, "t_end": 0.15,
}


def run_batched(rank: int, world: int):
    """Batched form against the plain form (one instance per launch) on the same seeded tubes.  The
    batched whole run is one persistent launch (each CTA runs tubes to their end, largest first);
    its step-synchronous form (one CUDA graph replay per RK3 step of the batch) gives the steady
    rate and a second whole-run figure.  Autotuned launch shape.  Instances are sharded over ranks;
    timing is max over ranks."""
    import torch

    import awcm
    from awcm import autotune, workloads
    from awcm.dist import reduce_run, shard_instances

    b_cfg = BATCHED
    tubes_all = workloads.shock_tubes(b_cfg["instances"])
    mine = shard_instances([t["nx"] for t in tubes_all], rank, world)
    tubes = [tubes_all[k] for k in mine]
    tol, cfl, t_end = b_cfg["tol"], b_cfg["cfl"], b_cfg["t_end"]
    best, rates = autotune.tune(lambda: workloads.make_batch(awcm, tubes), t_end, tol, cfl)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def fresh():
        bb = workloads.make_batch(awcm, tubes)
        bb.set_launch(*best)
        bb.set_run(tol, cfl, 0.0, t_end)
        bb.steps(3)
        bb.sync()
        return bb, bb.totals()[0], torch.cuda.ExternalStream(bb.stream)

    # Whole run: after 3 warm-up steps, one launch runs every tube to t_end (each CTA takes tubes
    # largest first and runs each one's steps back to back).
    b, u0, st = fresh()
    torch.cuda.synchronize()
    e0.record(st)
    b.run_all()
    e1.record(st)
    torch.cuda.synchronize()
    tot = b.totals()
    ms, upd = reduce_run(e0.elapsed_time(e1), tot[0] - u0, device="cuda")
    value = upd / (ms / 1e3)
    all_done = int(tot[2]) == b.n
    b.close()
    launches = 3 + 1
    # The same run as one graph replay per step of the whole batch (every tube one step a launch):
    # its first 250 steps are the steady rate, its whole run the step-synchronous figure.
    b, u0, st = fresh()
    torch.cuda.synchronize()
    e0.record(st)
    steady = None
    sw_launches = 3
    while True:
        b.steps(250)
        sw_launches += 250
        tot = b.totals()
        if steady is None:
            e1.record(st)
            torch.cuda.synchronize()
            steady = ((tot[0] - u0) / (e0.elapsed_time(e1) / 1e3))
        if tot[2] == b.n or sw_launches > 200000:
            break
    e1.record(st)
    torch.cuda.synchronize()
    sw_ms, sw_upd = reduce_run(e0.elapsed_time(e1), tot[0] - u0, device="cuda")
    b.close()
    # Plain form: one instance per launch.  (a) concurrent: each instance of a sample across the
    # size mix is its own batch of one (its own stream and graph), and every step launches each
    # unfinished instance separately, round robin over the streams, so the GPU runs as many
    # single-instance launches side by side as the host can issue; (b) serial: the same instances
    # one after the other on one stream.  Wall clock with the device synchronised on both sides.
    per_class = 8
    sample = []
    for J in sorted({t["jmax"] for t in tubes}):
        sample += [t for t in tubes if t["jmax"] == J][:per_class]
    plains = []
    for t in sample:
        p = workloads.make_batch(awcm, [t])
        p.set_launch(best[0], 0)
        p.set_run(tol, cfl, 0.0, t_end)
        p.steps(2)
        plains.append(p)
    for p in plains:
        p.sync()
    u0 = sum(p.totals()[0] for p in plains)
    live = list(plains)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    rounds = 0
    while live and time.perf_counter() - t0 < 4.0:
        for p in live:
            p.steps(1)
        rounds += 1
        if rounds % 64 == 0:
            live = [p for p in live if p.totals()[2] < 1]
    torch.cuda.synchronize()
    wall_c = time.perf_counter() - t0
    upd_c = sum(p.totals()[0] for p in plains) - u0
    for p in plains:
        p.close()
    conc_ms, conc_upd = reduce_run(wall_c * 1e3, upd_c, device="cuda")
    plain_conc = conc_upd / (conc_ms / 1e3)
    # (b) serial, one instance at a time on one stream, a sample of six across the mix
    serial = [sample[k] for k in range(0, len(sample), max(1, len(sample) // 6))][:6]
    p_ms, p_upd = 0.0, 0.0
    for t in serial:
        p = workloads.make_batch(awcm, [t])
        p.set_launch(best[0], 0)
        p.set_run(tol, cfl, 0.0, t_end)
        p.steps(3)
        p.sync()
        pu0 = p.totals()[0]
        pst = torch.cuda.ExternalStream(p.stream)
        torch.cuda.synchronize()
        e0.record(pst)
        t0 = time.perf_counter()
        while p.totals()[2] < 1 and time.perf_counter() - t0 < 2.0:
            p.steps(100)
        e1.record(pst)
        torch.cuda.synchronize()
        p_ms += e0.elapsed_time(e1)
        p_upd += p.totals()[0] - pu0
        p.close()
    p_ms, p_upd = reduce_run(p_ms, p_upd, device="cuda")
    plain_serial = p_upd / (p_ms / 1e3)
    return {
        "workload": b_cfg["workload"], "metric": METRIC, "value": value, "unit": UNIT,
        "steady_value": steady, "launches": launches, "instances": len(tubes_all), "ms": ms,
        "all_done": all_done,
        "stepwise": {"value": sw_upd / (sw_ms / 1e3), "ms": sw_ms, "launches": sw_launches,
                     "note": "the whole run as one launch per RK3 step of the batch (CUDA graph replays)"},
        "launch_shape": {"threads": best[0], "ctas_per_sm": best[1]},
        "autotune": {f"{k[0]}x{k[1]}": v for k, v in rates.items()},
        "plain": {"value": plain_conc, "unit": UNIT,
                  "sample": f"{len(sample)} instances ({per_class} per Jmax), each its own batch of one with its own "
                            "stream and graph; each step launches every unfinished instance separately, round robin "
                            "over the streams (one instance per launch, launches side by side); 4 s of wall clock"},
        "plain_serial": {"value": plain_serial, "unit": UNIT,
                         "sample": f"{len(serial)} of those instances one after another on one stream, up to 2 s each"},
        "batched_over_plain": value / plain_conc,
        "steady_over_plain": steady / plain_conc,
    }


GRADIENT = {
    "workload": "frozen-mask discrete adjoint: isentropic vortex (strength 5, radius 1) + 16 seeded density "
                "bumps on periodic [0,10]^2, 513x513 finest (17 coarse, 6 levels), eps 1e-3, 200 RK3 steps "
                "at dt = 0.4 dx / max(|u|+c+|v|+c), loss 1/2 |rho - target|^2 over mask0, sqrt(N) checkpoints, "
                "differentiable mode (WENO-Z eps 1e-6, smoothed |b0-b2| with delta 1e-6)",
    "num_levels": 6, "nx_coarse": 17, "tol": 1e-3, "steps": 200, "wenoz_eps": 1e-6, "tau_delta": 1e-6,
}


def run_adjoint(rank: int, world: int):
    """Reverse sweep (checkpoint recomputation included) against the frozen-mask forward run of
    the gradient workload; each rank runs one replica, times are max over ranks."""
    import awcm
    from awcm import gradient as G
    from awcm.dist import reduce_run

    c = GRADIENT
    s = awcm.AWCM2D(c["num_levels"], c["nx_coarse"], c["nx_coarse"], 0.0, 10.0, 0.0, 10.0,
                    bc_kind=awcm.BC_PERIODIC)
    q0 = G.vortex_bumps(s)
    target = G.target_density(s)
    dt = G.stable_dt(q0, 10.0 / (s.nx - 1))
    s.set_q(q0)
    s.prepare(c["tol"])
    s.set_wenoz(c["wenoz_eps"], c["tau_delta"])
    qp = s.get_q()
    n = c["steps"]
    s.adjoint(0.0, dt, n, target)  # warm-up; records the LF-speed tape
    fwd, rev, fwd_only, keep = [], [], [], []
    for _ in range(3):
        s.set_q(qp)
        loss, _, info = s.adjoint(0.0, dt, n, target, replay=True, with_grad=False)
        fwd.append(info["forward_ms"])
        rev.append(info["reverse_ms"])
        s.set_q(qp)
        fwd_only.append(s.frozen_run(0.0, dt, n, replay=True)[1])
    s.set_q(qp)
    _, _, kinfo = s.adjoint(0.0, dt, n, target, checkpoint_every=n, replay=True, with_grad=False)
    # gradient check: 16 seeded unit directions, central differences of the frozen replay
    s.set_q(qp)
    _, grad, _ = s.adjoint(0.0, dt, n, target, replay=True)
    act = G.active_points(s.get_masks())
    h = 1e-5
    rel = []
    for d in G.unit_directions(qp.shape, 16, 11):
        fd = []
        for sign in (1.0, -1.0):
            s.set_q(qp + sign * h * d)
            s.frozen_run(0.0, dt, n, replay=True)
            fd.append(s.get_q())
        fdv = G.loss_difference(fd[0], fd[1], target, act) / (2 * h)
        rel.append(abs(float((grad * d).sum()) - fdv) / abs(fdv))
    f_ms, _ = reduce_run(statistics.median(fwd), 0.0, device="cuda")
    r_ms, _ = reduce_run(statistics.median(rev), 0.0, device="cuda")
    fo_ms, _ = reduce_run(statistics.median(fwd_only), 0.0, device="cuda")
    k_ms, _ = reduce_run(kinfo["reverse_ms"], 0.0, device="cuda")
    m = s.get_masks()
    return {
        "workload": c["workload"], "steps": n, "dt": dt, "loss": loss,
        "checkpoint_every": info["checkpoint_every"], "device_bytes": info["device_bytes"],
        "forward_ms": fo_ms, "adjoint_forward_ms": f_ms, "reverse_ms": r_ms,
        "adjoint_over_forward": r_ms / fo_ms,
        "keep_all_reverse_ms": k_ms, "keep_all_over_forward": k_ms / fo_ms,
        "keep_all_device_bytes": kinfo["device_bytes"],
        "mask0_points": int(m[1, 3:-3, 3:-3].sum()), "mask3_points": int(m[4, 3:-3, 3:-3].sum()),
        "fd_check": {"directions": 16, "h": h, "max_rel": max(rel), "median_rel": statistics.median(rel)},
        "note": "forward = 200 frozen-mask steps replaying the LF speeds; reverse = the adjoint sweep "
                "including the recomputation of each checkpoint segment's stage inputs (device time, "
                "median of 3)",
    }


# --------------------------------------------------------------------- whole runs and late window
def make_2d(awcm, w):
    s = awcm.AWCM2D(w["num_levels"], w["nx_coarse"], w["ny_coarse"], *w["domain"], bc_kind=w.get("bc", 0))
    s.init_problem(w.get("problem", 0), *(w["split"] if "split" in w else (w["a"], w["b"])))
    return s


def timed_advance(torch, s, w, t, n):
    """n graph-replayed steps from t; device ms from CUDA events on the solver's stream."""
    st = torch.cuda.ExternalStream(s.stream)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(st)
    t, k, upd, _ = s.advance(w["tol"], w["cfl"], t, w["t_end"], n)
    e1.record(st)
    torch.cuda.synchronize()
    return t, k, upd, e0.elapsed_time(e1)


def whole_run(awcm, torch, w, save_at=None, path=None):
    """Workload w from its initial state to t_end in chunks of graph-replayed steps; device time
    summed over the chunks.  With save_at the state after exactly that many steps is written to
    `path` between two chunks (outside the timed chunks)."""
    warm = make_2d(awcm, w)
    warm.advance(w["tol"], w["cfl"], 0.0, w["t_end"], 2)  # graph and module load outside the timing
    warm.close()
    s = make_2d(awcm, w)
    t, steps, upd, ms, t_saved = 0.0, 0, 0.0, 0.0, None
    while t < w["t_end"]:
        n = 256 if not save_at or steps >= save_at else min(256, save_at - steps)
        t, k, u, dms = timed_advance(torch, s, w, t, n)
        steps, upd, ms = steps + k, upd + u, ms + dms
        if save_at and steps == save_at and t_saved is None:
            s.save_state(path, t, steps)
            t_saved = t
        if k < n:
            break
    s.close()
    return {"value": upd / (ms / 1e3), "unit": UNIT, "steps": steps, "t_end": t, "device_ms": ms,
            "active_points": upd, "ms_per_step": ms / max(1, steps)}, t_saved


def run_full_and_late(awcm, torch, args, cpu_ok):
    """The headline workload's whole run to t_end, and a late window: the GPU and the reference's
    own code each time the steps after the same mid-run state (written by the whole run)."""
    w = WORKLOAD
    fd, path = tempfile.mkstemp(suffix=".awcmstate")
    os.close(fd)
    try:
        full, t_late = whole_run(awcm, torch, w, save_at=LATE_STEP, path=path)
        full["note"] = ("whole run of the headline workload from its initial state to t_end, graph-replayed "
                        "steps in chunks of 256, device time (CUDA events) summed over the chunks")
        late = None
        if t_late is not None:
            s = make_2d(awcm, w)
            s.advance(w["tol"], w["cfl"], 0.0, w["t_end"], 1)  # graph built before the state is loaded
            s.load_state(path)
            _, k, upd, ms = timed_advance(torch, s, w, t_late, args.steps)
            m = s.get_masks()
            late = {"first_step": LATE_STEP + 1, "last_step": LATE_STEP + k, "t_start": t_late,
                    "gpu": {"value": upd / (ms / 1e3), "unit": UNIT, "steps": k, "ms_per_step": ms / max(1, k),
                            "active_points_per_step": upd / max(1, k)},
                    "mask3_points": int(m[4, 3:-3, 3:-3].sum())}
            s.close()
            if cpu_ok:
                r, why = time_reference(args.steps, args.cpu_seconds, w=w, state_file=path, t0_run=t_late)
                if r is not None:
                    late["reference"] = {"value": r["value"], "unit": UNIT, "cores": r["cores"], "kind": "reference",
                                         "steps": r["steps"], "ms_per_step": 1e3 * r["wall_s"] / r["steps"],
                                         "sample": f"steps {LATE_STEP + 1}..{LATE_STEP + r['steps']} from the GPU "
                                                   f"run's state file at step {LATE_STEP} (OpenMP)"}
                    late["gpu_over_reference"] = late["gpu"]["value"] / r["value"]
                else:
                    late["reference"] = {"value": None, "sample": why}
        return {"full_run": full, "late_window": late}
    finally:
        try:
            os.unlink(path)
        except OSError:
            pass


def run_configs(awcm, torch, args, warmup, cpu_ok):
    """The double-Mach (4097x1025) and 1D Sod configurations beside the headline: GPU and the
    reference's own code on the same steps."""
    out = {}
    # double Mach: the headline's window (W warm-up steps, K timed) and the whole run to t_end
    w = DOUBLE_MACH
    s = make_2d(awcm, w)
    t, _, _, _ = s.advance(w["tol"], w["cfl"], 0.0, w["t_end"], warmup)
    _, k, upd, ms = timed_advance(torch, s, w, t, args.steps)
    s.close()
    full, _ = whole_run(awcm, torch, w)
    dm = {"workload": w["workload"], "metric": METRIC,
          "window": {"first_step": warmup + 1, "last_step": warmup + k},
          "value": upd / (ms / 1e3), "unit": UNIT, "ms_per_step": ms / max(1, k), "full_run": full}
    if cpu_ok:
        r, why = time_reference(args.steps, args.cpu_seconds, warmup=warmup, w=w)
        if r is not None:
            dm["cpu_baseline"] = {"value": r["value"], "unit": UNIT, "cores": r["cores"], "kind": "reference",
                                  "sample": f"steps {warmup + 1}..{warmup + r['steps']} from the initial state "
                                            f"(OpenMP), the GPU's window"}
            dm["gpu_over_reference"] = dm["value"] / r["value"]
    out["double_mach_4097x1025"] = dm
    # 1D Sod: one instance, whole run to t_end (897 steps)
    c = SOD
    n = c["n"]
    geo = (c["num_levels"], c["nx_coarse"], 0.5 / n, 1 - 0.5 / n)
    warm = awcm.AWCM1D(*geo)
    warm.init_riemann(0.5, (1.0, 0.0, 1.0), (0.125, 0.0, 0.1))
    warm.run(c["tol"], c["cfl"], c["t_end"])
    warm.b.close()
    g = awcm.AWCM1D(*geo)
    g.init_riemann(0.5, (1.0, 0.0, 1.0), (0.125, 0.0, 0.1))
    st = torch.cuda.ExternalStream(g.b.stream)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(st)
    steps, t, upd = g.run(c["tol"], c["cfl"], c["t_end"])
    e1.record(st)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    sod = {"workload": c["workload"], "metric": METRIC, "value": upd / (ms / 1e3), "unit": UNIT, "steps": steps,
           "device_ms": ms, "active_points": upd,
           "note": "one instance on one CTA (the batch kernel with a batch of one), the whole run in one launch"}
    g.b.close()
    if cpu_ok:
        import oracle

        if oracle.reference_available():
            o = oracle.Oracle1D(*geo, kind="reference")
            o.init_riemann(0.5, (1.0, 0.0, 1.0), (0.125, 0.0, 0.1))
            t0 = time.perf_counter()
            n_r, _, u_r = o.run(c["tol"], c["cfl"], c["t_end"])
            wall = time.perf_counter() - t0
            sod["cpu_baseline"] = {"value": u_r / wall, "unit": UNIT, "cores": 1, "kind": "reference",
                                   "steps": n_r, "sample": "the whole run, the reference's serial 1D code"}
            sod["gpu_over_reference"] = sod["value"] / (u_r / wall)
    out["sod_1d_1025"] = sod
    return out


# ------------------------------------------------------------------------------------- GPU arm
def run_b200(args):
    rank, world, local = dist_env()
    import numpy as np
    import torch

    if not torch.cuda.is_available():
        raise SystemExit("bench.py: no CUDA device")
    torch.cuda.set_device(local)
    if world > 1:
        import torch.distributed as dist

        dist.init_process_group("nccl", device_id=torch.device("cuda", local))
    import awcm

    w = WORKLOAD
    s = awcm.AWCM2D(w["num_levels"], w["nx_coarse"], w["ny_coarse"], *w["domain"], bc_kind=0)
    s.init_problem(0, *w["split"])
    stream = torch.cuda.ExternalStream(s.stream)
    tol, cfl, t_end = w["tol"], w["cfl"], w["t_end"]
    launches = s.launches_per_step()

    def barrier():
        torch.cuda.synchronize()
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()

    from awcm.dist import reduce_run

    warmup = max(3, args.warmup)
    t, n, _, _ = s.advance(tol, cfl, 0.0, t_end, warmup)
    t_after_warmup = t

    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        barrier()
        e0.record(stream)
        t, n_steps, upd, stage_pts = s.advance(tol, cfl, t, t_end, args.steps)
        e1.record(stream)
        barrier()
    ms = e0.elapsed_time(e1)
    ms_max, upd_all = reduce_run(ms, upd, device="cuda")
    value = upd_all / (ms_max / 1e3)
    clocks = clk.summary()

    # Roofline of the dominant kernel (the WENO-Z/Roe face flux): profiled steps with CUDA events
    # around the face kernels on the solver's stream, same kernels as the graph.
    prof = []
    for _ in range(3):
        prof.append(s.profile_step(tol, cfl, t, t_end))
        t += prof[-1]["dt"]
    face_ms = sum(sum(p["face_ms"]) for p in prof)
    faces = sum(sum(p["faces"]) for p in prof)
    step_ms = sum(p["total_ms"] for p in prof)
    achieved = faces * FLOPS_PER_FACE / (face_ms * 1e-3) / 1e12
    peak = awcm.measure_fp64_peak()
    phase = {k: (sum(p[k] for p in prof) / len(prof) if not isinstance(prof[0][k], list)
                 else [sum(p[k][i] for p in prof) / len(prof) for i in range(3)])
             for k in ("prepare_ms", "setup_ms", "face_ms", "update_ms", "between_ms", "post_ms", "total_ms")}
    traffic = None
    tr_path = os.path.join(ROOT, "profiles", "face_flux_traffic.json")
    if os.path.exists(tr_path):
        try:
            per_face = json.load(open(tr_path))["dram_bytes_per_face"]
            traffic = per_face * faces / (len(prof) * 6)
        except Exception:
            traffic = None

    # End to end through the public C-ABI with host buffers: every step uploads the conserved
    # field in the reference's host layout from pinned memory, advances one step and reads it back.
    e2e = None
    e2e_field = None
    if not args.no_e2e:
        # (a) the driver loop as a user writes it: one synchronous awcm2d_step per RK3 step (step
        # parameters host -> device, the step's results dt / output flag / mask sizes device ->
        # host), the state staying resident on the GPU as it does between the reference's steps.
        h2d_b, d2h_b = ctypes.c_longlong(), ctypes.c_longlong()
        awcm._lib.call("awcm2d_step_io_bytes", s.h, ctypes.byref(h2d_b), ctypes.byref(d2h_b))
        n_step = max(5, min(args.steps, 40))
        barrier()
        t0 = time.perf_counter()
        upd_s = 0.0
        for _ in range(n_step):
            o = s.step(tol, cfl, t, t_end)
            upd_s += o[2]
            t += o[0]
        barrier()
        wall_s, upd_s_all = reduce_run(time.perf_counter() - t0, upd_s, device="cuda")
        e2e = {"value": upd_s_all / wall_s, "unit": UNIT, "h2d_bytes_per_step": h2d_b.value,
               "d2h_bytes_per_step": d2h_b.value, "steps": n_step,
               "note": "wall clock of synchronous awcm2d_step calls (the public per-step C-ABI call): step "
                       "parameters in, dt / output flag / mask sizes out, state resident on the GPU"}
        # (b) the same with the whole conserved field handed over in the reference's host layout
        # every step (a driver that keeps Q on the host).
        shape = (s.ny + 6, s.nx + 6, 4)
        host_in = torch.empty(shape, dtype=torch.float64, pin_memory=True)
        host_out = torch.empty(shape, dtype=torch.float64, pin_memory=True)
        host_in.numpy()[...] = s.get_q()
        n_e2e = max(3, min(args.steps, 10))
        barrier()
        t0 = time.perf_counter()
        upd_e = 0.0
        for _ in range(n_e2e):
            awcm._lib.call("awcm2d_set_q", s.h, awcm._lib.ptr(host_in.numpy(), ctypes.c_double))
            t, k, u, _ = s.advance(tol, cfl, t, t_end, 1)
            upd_e += u
            awcm._lib.call("awcm2d_get_q", s.h, awcm._lib.ptr(host_out.numpy(), ctypes.c_double))
            host_in, host_out = host_out, host_in
        barrier()
        wall, upd_e_all = reduce_run(time.perf_counter() - t0, upd_e, device="cuda")
        nbytes = int(np.prod(shape)) * 8
        e2e_field = {"value": upd_e_all / wall, "unit": UNIT, "h2d_bytes_per_step": nbytes,
                     "d2h_bytes_per_step": nbytes, "steps": n_e2e,
                     "note": "per step: H2D of the dense conserved field (reference layout, pinned), one RK3 "
                             "step, D2H of the field"}

    cpu = None
    cpu_ok = rank == 0 and world == 1 and not args.no_cpu_baseline
    if cpu_ok:
        # the same step window as the timed GPU steps: W untimed warm-up steps, then steps W+1 ..
        r, why = time_reference(args.steps, args.cpu_seconds, warmup=warmup)
        if r is not None:
            cpu = {"value": r["value"], "unit": UNIT, "cores": r["cores"], "kind": "reference",
                   "window": {"first_step": warmup + 1, "last_step": warmup + r["steps"]},
                   "sample": f"steps {warmup + 1}..{warmup + r['steps']} of the same 2049^2 workload from its "
                             f"initial state, the GPU's timed window ({r['wall_s']:.1f} s, reference code "
                             f"compiled from the reference tree, OpenMP)"}
        else:
            cpu = {"value": None, "unit": UNIT, "cores": 0, "kind": "reference", "sample": why}

    full = None if args.no_full_run else run_full_and_late(awcm, torch, args, cpu_ok)
    configs = None if args.no_configs else run_configs(awcm, torch, args, warmup, cpu_ok)
    batched = None if args.no_batched else run_batched(rank, world)
    gradient = None if args.no_adjoint else run_adjoint(rank, world)

    pitch = (s.nx + 6 + 31) // 32 * 32
    state_bytes = 5 * 4 * 8 * pitch * (s.ny + 6)  # Q, Q2, Q1, Fx, Fy planes
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": n_steps, "warmup": warmup,
        "ms_per_step": ms_max / max(1, n_steps), "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic (deterministic four-quadrant initial state, no dataset)",
        "config": dict(WORKLOAD, parallelism=f"replicas{world}" if world > 1 else "single GPU",
                       l2="no flush: device state %.0f MB > 126 MB L2" % (state_bytes / 1e6),
                       steps_from=f"after {warmup} warm-up steps from t=0 (t={t_after_warmup:.3e})"),
        "roofline": {"bound": "fp64", "kernel": "k_face (WENO-Z/Roe face flux)", "achieved": achieved,
                     "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak, "traffic": traffic,
                     "peak_note": "of measured: dense DFMA probe on this GPU (2 flops per FMA)",
                     "flops_per_face": FLOPS_PER_FACE, "faces_per_step": faces / len(prof),
                     "face_ms_per_step": face_ms / len(prof)},
        "phase_ms_per_step": phase,
        "active_points_per_step": upd_all / max(1, n_steps) / world,
        "stage_points_per_step": stage_pts / max(1, n_steps),
        "clocks": clocks,
        "e2e": e2e,
        "e2e_field_roundtrip": e2e_field,
        "cpu_baseline": cpu,
        "window": {"first_step": warmup + 1, "last_step": warmup + n_steps},
        "full_run": full["full_run"] if full else None,
        "late_window": full["late_window"] if full else None,
        "configs": configs,
        "batched_1d": batched,
        "adjoint": gradient,
        "gpu_launches": launches * n_steps,
        "launches_per_step": launches,
    }
    if rank == 0:
        print(json.dumps(line))
    if world > 1:
        torch.distributed.destroy_process_group()


def run_capture(k: int):
    """Small, self-ending run for ncu: the benchmark instance, k graph-replayed steps and one
    profiled step (its face kernels are launches 6k+1 .. 6k+6 of k_face)."""
    import awcm

    w = WORKLOAD
    s = awcm.AWCM2D(w["num_levels"], w["nx_coarse"], w["ny_coarse"], *w["domain"], bc_kind=0)
    s.init_problem(0, *w["split"])
    t, _, _, _ = s.advance(w["tol"], w["cfl"], 0.0, w["t_end"], k)
    print(json.dumps(s.profile_step(w["tol"], w["cfl"], t, w["t_end"])))


def run_capture_batch(k: int, skip: int = 0):
    """Small, self-ending run for ncu: the seeded 512-tube batch at 768 threads per CTA, `skip` RK3
    steps, then k more (each step one k_step1d launch), then its totals and the running instances."""
    import awcm
    from awcm import workloads

    b = workloads.make_batch(awcm, workloads.shock_tubes(BATCHED["instances"]))
    b.set_launch(768, 0)
    b.set_run(BATCHED["tol"], BATCHED["cfl"], 0.0, BATCHED["t_end"])
    if skip:
        b.steps(skip)
        b.sync()
    live = [i for i in range(b.n) if b.status(i)[3] == 0]
    b.steps(k)
    b.sync()
    print(json.dumps({"skip": skip, "steps": k, "running_before": len(live), "running": live[:16],
                      "totals": b.totals().tolist()}))


def main():
    args = parse()
    if args.capture >= 0:
        run_capture(args.capture)
        return
    if args.capture_batch >= 0:
        run_capture_batch(args.capture_batch, args.capture_skip)
        return
    if args.impl == "reference":
        run_reference_arm(args)
    else:
        run_b200(args)


if __name__ == "__main__":
    main()
