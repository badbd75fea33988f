"""Test infrastructure only: the binary 2D state file, read and written on the CPU side.

The same layout as the product's awcm2d_save_state / awcm2d_load_state, restated with numpy and
the standard-library CRC-32 (zlib.crc32, the IEEE 802.3 reflected polynomial):

  header (128 bytes, little-endian): magic "AWCMST2D", uint32 version (1), uint32 header bytes
  (128), int32 num_levels, nx_coarse, ny_coarse, nx, ny, bc_kind, float64 x_min, x_max, y_min,
  y_max, gamma, t, int64 step, uint64 |mask0|, uint64 payload bytes, uint32 CRC-32 of the payload,
  zero padding;
  payload: 5 mask planes (mask_temp, mask0..mask3) over the ghosted (Ny+6) x (Nx+6) points, one
  bit per point, least significant bit first, each plane padded to whole bytes; 4 level planes
  over the Nx x Ny points, one signed byte each; (rho, rho u, rho v, E) of the mask0 grid points in
  row-major order.

The checker uses it to hand states to and from the CUDA path (cross-tool parity) and to check
the product's files.
"""
from __future__ import annotations

import struct
import zlib

import numpy as np

MAGIC = b"AWCMST2D"
VERSION = 1
HEADER_BYTES = 128
_HEAD = struct.Struct("<8sII6i6dqQQI")


def write_state(path, geometry, q, masks, levels, t, step):
    """geometry = (num_levels, nx_coarse, ny_coarse, bc_kind, x_min, x_max, y_min, y_max, gamma);
    q (Ny+6, Nx+6, 4), masks (5, Ny+6, Nx+6), levels (4, Ny, Nx)."""
    nl, nxc, nyc, bc, x0, x1, y0, y1, gamma = geometry
    q = np.asarray(q, np.float64)
    ny, nx = q.shape[0] - 6, q.shape[1] - 6
    m = np.asarray(masks, np.uint8).reshape(5, -1) != 0
    planes = b"".join(np.packbits(m[p], bitorder="little").tobytes() for p in range(5))
    lv = np.asarray(levels).astype(np.int8).tobytes()
    on = m[1].reshape(ny + 6, nx + 6)[3:-3, 3:-3]
    vals = np.ascontiguousarray(q[3:-3, 3:-3][on]).tobytes()
    payload = planes + lv + vals
    head = _HEAD.pack(MAGIC, VERSION, HEADER_BYTES, int(nl), int(nxc), int(nyc), nx, ny, int(bc), x0, x1, y0, y1,
                      gamma, t, int(step), int(on.sum()), len(payload), zlib.crc32(payload) & 0xFFFFFFFF)
    with open(path, "wb") as f:
        f.write(head.ljust(HEADER_BYTES, b"\0"))
        f.write(payload)


def read_state(path):
    """Returns dict(geometry, nx, ny, t, step, q, masks, levels); raises ValueError on a bad file."""
    raw = open(path, "rb").read()
    if len(raw) < HEADER_BYTES:
        raise ValueError("truncated header")
    (magic, ver, hb, nl, nxc, nyc, nx, ny, bc, x0, x1, y0, y1, gamma, t, step, n_act, n_pay,
     crc) = _HEAD.unpack_from(raw, 0)
    if magic != MAGIC or ver != VERSION or hb != HEADER_BYTES:
        raise ValueError("not an AWCM 2D state file of version 1")
    payload = raw[HEADER_BYTES:]
    ng, ni = (nx + 6) * (ny + 6), nx * ny
    pb = (ng + 7) // 8
    if len(payload) != n_pay or n_pay != 5 * pb + ni * 4 + n_act * 32:
        raise ValueError("payload size does not match the header")
    if zlib.crc32(payload) & 0xFFFFFFFF != crc:
        raise ValueError("payload CRC-32 mismatch")
    masks = np.stack([np.unpackbits(np.frombuffer(payload[p * pb:(p + 1) * pb], np.uint8), bitorder="little")[:ng]
                      for p in range(5)]).reshape(5, ny + 6, nx + 6)
    off = 5 * pb
    levels = np.frombuffer(payload[off:off + 4 * ni], np.int8).astype(np.int32).reshape(4, ny, nx)
    off += 4 * ni
    vals = np.frombuffer(payload[off:], np.float64).reshape(-1, 4)
    q = np.zeros((ny + 6, nx + 6, 4))
    on = masks[1, 3:-3, 3:-3].astype(bool)
    if int(on.sum()) != n_act:
        raise ValueError("mask0 size differs from the stored value count")
    inner = q[3:-3, 3:-3]
    inner[on] = vals
    return dict(geometry=(nl, nxc, nyc, bc, x0, x1, y0, y1, gamma), nx=nx, ny=ny, t=t, step=step, q=q,
                masks=masks, levels=levels)
