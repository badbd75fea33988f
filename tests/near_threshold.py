"""Near-threshold report of the mask parity rule: the points whose wavelet detail lies within
1e-12 relative of the threshold are counted separately, because there the keep/drop decision of
the threshold test (WAVELET_2D.h:530, |d| < tol) hangs on the last bits of the detail.

The details come from the CPU restatement's forward transform with threshold 0 (no point is
dropped, and the detail values do not depend on the threshold).
"""
from __future__ import annotations

import numpy as np

from oracle import Oracle2D


def detail_ratios(geom, q, masks, tol):
    """|d| / tol at the active detail points of the state (q, masks) on the grid `geom`
    = (num_levels, nx_coarse, ny_coarse, x_min, x_max, y_min, y_max, bc_kind)."""
    nl, nxc, nyc, x0, x1, y0, y1, bc = geom
    o = Oracle2D(nl, nxc, nyc, x0, x1, y0, y1, bc_kind=bc, kind="port")
    o.set_q(q)
    o.set_masks(masks)
    o.fwt(0.0)
    d = o.get_q()[3:-3, 3:-3, 0]
    on = masks[1, 3:-3, 3:-3].astype(bool)
    ny, nx = on.shape
    D = 1 << (nl - 1)
    coarse = (np.arange(ny)[:, None] % D == 0) & (np.arange(nx)[None, :] % D == 0)
    sel = on & ~coarse
    return np.abs(d[sel]) / tol


def near_threshold(geom, q, masks, tol, rel=1e-12):
    """(points within `rel` of the threshold, active detail points examined)."""
    r = detail_ratios(geom, q, masks, tol)
    return int(np.count_nonzero(np.abs(r - 1.0) <= rel)), int(r.size)
