"""Launch-shape autotuner of the batched 1D step kernel.

The step kernel runs one instance per CTA, with up to 768 threads (80 registers a thread); the CTA
size trades occupancy (CTAs resident per SM, i.e. instances in flight) against per-instance
parallelism.  The tuner times a few RK3 steps of the actual batch for each candidate shape on a
throw-away copy of the batch and keeps the fastest (active-point updates per second)."""
from __future__ import annotations

import time

CANDIDATES = [(128, 0), (256, 0), (384, 0), (512, 0), (640, 0), (768, 0), (128, 2), (256, 2)]


def tune(make_copy, t_end: float, tol: float = 1e-4, cfl: float = 0.5, steps: int = 40, candidates=CANDIDATES):
    """make_copy() -> fresh AWCM1DBatch at its initial state.  Returns (best (threads, ctas_per_sm),
    {shape: updates/s})."""
    import torch

    rates = {}
    from ._lib import AwcmError

    for shape in candidates:
        b = make_copy()
        try:
            b.set_launch(*shape)
        except AwcmError:  # more threads than the kernel's registers allow
            b.close()
            continue
        b.set_run(tol, cfl, 0.0, t_end)
        b.steps(3)  # warm-up (also builds the graph)
        b.sync()
        u0 = b.totals()[0]
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        b.steps(steps)
        b.sync()
        dt = time.perf_counter() - t0
        rates[shape] = (b.totals()[0] - u0) / dt
        b.close()
    best = max(rates, key=rates.get)
    return best, rates
