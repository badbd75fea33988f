"""Physical sanity of the 1D Sod configuration (not parity): the oracle's density at t = 0.2 is
close to the exact Riemann solution.  The exact solver follows Toro, "Riemann Solvers and
Numerical Methods for Fluid Dynamics", ch. 4: Newton iteration on the star pressure, then sampling
of the self-similar solution."""
import math

import numpy as np

from oracle import Oracle1D

G = 1.4


def _f(p, rho, pk, ck):
    if p > pk:  # shock
        a, b = 2 / ((G + 1) * rho), (G - 1) / (G + 1) * pk
        return (p - pk) * math.sqrt(a / (p + b)), math.sqrt(a / (b + p)) * (1 - 0.5 * (p - pk) / (b + p))
    r = p / pk  # rarefaction
    return 2 * ck / (G - 1) * (r ** ((G - 1) / (2 * G)) - 1), 1 / (rho * ck) * r ** (-(G + 1) / (2 * G))


def exact_density(x, t, x0, L, R):
    rl, ul, pl = L
    rr, ur, pr = R
    cl, cr = math.sqrt(G * pl / rl), math.sqrt(G * pr / rr)
    p = 0.5 * (pl + pr)
    for _ in range(100):
        fl, dl = _f(p, rl, pl, cl)
        fr, dr = _f(p, rr, pr, cr)
        dp = (fl + fr + ur - ul) / (dl + dr)
        p = max(p - dp, 1e-12)
        if abs(dp) < 1e-14 * p:
            break
    fl, _ = _f(p, rl, pl, cl)
    fr, _ = _f(p, rr, pr, cr)
    u = 0.5 * (ul + ur) + 0.5 * (fr - fl)
    out = np.empty_like(x)
    for k, xv in enumerate(x):
        s = (xv - x0) / t
        if s <= u:  # left of contact
            if p > pl:
                sl = ul - cl * math.sqrt((G + 1) / (2 * G) * p / pl + (G - 1) / (2 * G))
                out[k] = rl if s < sl else rl * ((p / pl + (G - 1) / (G + 1)) / ((G - 1) / (G + 1) * p / pl + 1))
            else:
                csl = cl * (p / pl) ** ((G - 1) / (2 * G))
                if s < ul - cl:
                    out[k] = rl
                elif s > u - csl:
                    out[k] = rl * (p / pl) ** (1 / G)
                else:
                    out[k] = rl * (2 / (G + 1) + (G - 1) / ((G + 1) * cl) * (ul - s)) ** (2 / (G - 1))
        else:
            if p > pr:
                sr = ur + cr * math.sqrt((G + 1) / (2 * G) * p / pr + (G - 1) / (2 * G))
                out[k] = rr if s > sr else rr * ((p / pr + (G - 1) / (G + 1)) / ((G - 1) / (G + 1) * p / pr + 1))
            else:
                csr = cr * (p / pr) ** ((G - 1) / (2 * G))
                if s > ur + cr:
                    out[k] = rr
                elif s < u + csr:
                    out[k] = rr * (p / pr) ** (1 / G)
                else:
                    out[k] = rr * (2 / (G + 1) - (G - 1) / ((G + 1) * cr) * (ur - s)) ** (2 / (G - 1))
    return out


def test_sod_density_near_exact_solution():
    n = 1025
    o = Oracle1D(7, 17, 0.5 / n, 1 - 0.5 / n, kind="port")
    o.init_riemann(0.5, (1.0, 0.0, 1.0), (0.125, 0.0, 0.1))
    steps, t, _ = o.run(1e-4, 0.5, 0.2)
    assert abs(t - 0.2) < 1e-12
    x = 0.5 / n + np.arange(n) / n
    rho = o.get_q()[3:-3, 0]
    active = o.get_masks()[1, 3:-3].astype(bool)
    ex = exact_density(x, 0.2, 0.5, (1.0, 0.0, 1.0), (0.125, 0.0, 0.1))
    err = np.abs(rho[active] - ex[active])
    assert np.mean(err) < 5e-3, np.mean(err)
    assert np.median(err) < 1e-4
