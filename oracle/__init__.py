"""Test infrastructure only: ctypes front-end to the two CPU checkers.

* ``Oracle1D/Oracle2D(kind="port")`` drive the CPU restatement (``awcm_oracle.cpp``, built into
  ``oracle/_build/libawcm_oracle.so``).
* ``Oracle1D/Oracle2D(kind="reference")`` drive the reference's own AWCM code compiled from the
  reference tree behind ``ref_harness_1d.cpp`` / ``ref_harness_2d.cpp`` (``oracle/_ref/*.so``).

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline / reference arms
use this package, and only as the checker or the timed CPU baseline; the product never does.

Layouts (host, ghost ring of 3):
  1D state  (Nx+6, 3) float64
  2D state  (Ny+6, Nx+6, 4) float64
  masks     (5, ...) uint8 planes: mask_temp, mask0, mask1, mask2, mask3
  levels    (4, ...) int32 planes: level0..level3 (interior points only)
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PORT_LIB = os.path.join(HERE, "_build", "libawcm_oracle.so")
REF_LIB_1D = os.path.join(HERE, "_ref", "libawcm_ref1d.so")
REF_LIB_2D = os.path.join(HERE, "_ref", "libawcm_ref2d.so")


def reference_tree() -> str:
    """Location of the reference source tree: $AWCM_REFERENCE_TREE, else the default of the build
    recipe (oracle/Makefile, variable REF).  The tree is read only to build oracle/_ref."""
    env = os.environ.get("AWCM_REFERENCE_TREE")
    if env:
        return env
    try:
        r = subprocess.run(["make", "-s", "--no-print-directory", "-C", HERE, "print-ref"], capture_output=True,
                           text=True, timeout=30)
        return r.stdout.strip()
    except Exception:
        return ""

# manager op codes shared by both checkers and by the product's C-ABI
AAZ, CR, APD, CL, RR, BAND = 0, 1, 2, 3, 4, 5

_c_int, _c_double, _vp = ctypes.c_int, ctypes.c_double, ctypes.c_void_p
_dp = ctypes.POINTER(ctypes.c_double)


def build(with_reference: bool | None = None) -> None:
    """Compiles the restatement, and the reference harness when the reference tree exists."""
    targets = ["oracle"]
    tree = reference_tree()
    if with_reference is None:
        with_reference = bool(tree) and os.path.isdir(tree)
    if with_reference:
        targets.append("ref")
    subprocess.run(["make", "-s", "-C", HERE] + targets + ([f"REF={tree}"] if tree else []), check=True)


def reference_available() -> bool:
    return os.path.exists(REF_LIB_1D) and os.path.exists(REF_LIB_2D)


_libs: dict[str, ctypes.CDLL] = {}


def _load(path: str) -> ctypes.CDLL:
    if path not in _libs:
        if not os.path.exists(path):
            raise FileNotFoundError(f"checker library missing: {path} (run make -C oracle)")
        _libs[path] = ctypes.CDLL(path)
    return _libs[path]


def _ptr(a: np.ndarray, ctype):
    return a.ctypes.data_as(ctypes.POINTER(ctype))


def _bind(lib, name, restype, argtypes):
    f = getattr(lib, name)
    f.restype = restype
    f.argtypes = argtypes
    return f


class Oracle1D:
    """One 1D AWCM Euler instance on the CPU (restatement or the reference itself)."""

    def __init__(self, num_levels: int, nx_coarse: int, x_min: float, x_max: float,
                 gamma: float = 1.4, scheme: int = 0, kind: str = "port"):
        self.kind = kind
        lib = _load(PORT_LIB if kind == "port" else REF_LIB_1D)
        p = "or1d_" if kind == "port" else "ref1d_"
        b = lambda n, r, a: _bind(lib, p + n, r, a)
        self._create = b("create", _vp, [_c_int, _c_int, _c_double, _c_double, _c_double, _c_int])
        self._destroy = b("destroy", None, [_vp])
        self._nx = b("nx", _c_int, [_vp])
        self._set_q = b("set_q", None, [_vp, _dp])
        self._get_q = b("get_q", None, [_vp, _dp])
        self._init_riemann = b("init_riemann", None, [_vp] + [_c_double] * 7)
        self._get_masks = b("get_masks", None, [_vp, ctypes.POINTER(ctypes.c_uint8)])
        self._set_masks = b("set_masks", None, [_vp, ctypes.POINTER(ctypes.c_uint8)])
        self._get_levels = b("get_levels", None, [_vp, ctypes.POINTER(ctypes.c_int)])
        self._set_levels = b("set_levels", None, [_vp, ctypes.POINTER(ctypes.c_int)])
        self._prepare = b("prepare", None, [_vp, _c_double])
        self._fwt = b("fwt", None, [_vp, _c_double])
        self._iwt = b("iwt", None, [_vp, _c_int])
        self._manager = b("manager", None, [_vp, _c_int, _c_int, _c_int])
        self._step = b("step", None, [_vp, _c_double, _c_double, _c_double, _c_double, _dp])
        self._run = b("run", _c_int, [_vp, _c_double, _c_double, _c_double, _c_int, _dp])
        self._scalar_step = b("scalar_step", None, [_vp, _c_double, _c_double, _dp])
        self._interpolate = b("interpolate", None, [_vp, _c_int, _c_int])
        self._apply_bc = b("apply_bc", None, [_vp])
        self._set_bc_field = b("set_bc_field", None, [_vp, ctypes.POINTER(_c_int)])
        self.h = self._create(num_levels, nx_coarse, x_min, x_max, gamma, scheme)
        self.nx = self._nx(self.h)

    def __del__(self):
        if getattr(self, "h", None):
            self._destroy(self.h)
            self.h = None

    def set_q(self, q):
        q = np.ascontiguousarray(q, dtype=np.float64).reshape(self.nx + 6, 3)
        self._set_q(self.h, _ptr(q, ctypes.c_double))

    def get_q(self):
        q = np.empty((self.nx + 6, 3), np.float64)
        self._get_q(self.h, _ptr(q, ctypes.c_double))
        return q

    def init_riemann(self, x_interface, left, right):
        self._init_riemann(self.h, x_interface, *left, *right)

    def get_masks(self):
        m = np.empty((5, self.nx + 6), np.uint8)
        self._get_masks(self.h, _ptr(m, ctypes.c_uint8))
        return m

    def set_masks(self, m):
        m = np.ascontiguousarray(m, dtype=np.uint8).reshape(5, self.nx + 6)
        self._set_masks(self.h, _ptr(m, ctypes.c_uint8))

    def get_levels(self):
        lv = np.empty((4, self.nx), np.int32)
        self._get_levels(self.h, _ptr(lv, ctypes.c_int))
        return lv

    def set_levels(self, lv):
        lv = np.ascontiguousarray(lv, dtype=np.int32).reshape(4, self.nx)
        self._set_levels(self.h, _ptr(lv, ctypes.c_int))

    def prepare(self, tol):
        self._prepare(self.h, tol)

    def fwt(self, tol):
        self._fwt(self.h, tol)

    def iwt(self, mask_id=3):
        self._iwt(self.h, mask_id)

    def manager(self, op, mask_id, level_id=0):
        self._manager(self.h, op, mask_id, level_id)

    def interpolate(self, from_id=4, to_id=3):
        """WAVELET_1D::InterpolateEuler(Q, mra, mask_from, mask_to)."""
        self._interpolate(self.h, from_id, to_id)

    def apply_bc(self):
        """The ghost fill: transmissive BOUNDARY_MANAGER, or the generic one once attached."""
        self._apply_bc(self.h)

    def set_bc_field(self, bc):
        """Attaches BOUNDARY_MANAGER_1D<T> with the BOUNDARY_CONDITION field bc (Nx+6 ints)."""
        bc = np.ascontiguousarray(bc, dtype=np.int32).reshape(self.nx + 6)
        self._set_bc_field(self.h, _ptr(bc, ctypes.c_int))

    def step(self, tol, cfl, t, t_next):
        out = np.zeros(10)
        self._step(self.h, tol, cfl, t, t_next, _ptr(out, ctypes.c_double))
        return out

    def run(self, tol, cfl, t_end, max_steps=1 << 30):
        out = np.zeros(2)
        n = self._run(self.h, tol, cfl, t_end, max_steps, _ptr(out, ctypes.c_double))
        return n, out[0], out[1]

    def scalar_step(self, tol, dt):
        """Scheme 2 (the scalar path of Wavelet/main_1d_advect.cpp): one driver pass at the fixed dt;
        returns [dt, |mask0|, |mask1|, |mask2|, |mask3|].  The field is column 0 of set_q/get_q."""
        out = np.zeros(5)
        self._scalar_step(self.h, tol, dt, _ptr(out, ctypes.c_double))
        return out


class Oracle2D:
    """One 2D AWCM Euler instance on the CPU (restatement or the reference itself)."""

    def __init__(self, num_levels: int, nx_coarse: int, ny_coarse: int, x_min: float, x_max: float,
                 y_min: float, y_max: float, bc_kind: int = 0, kind: str = "port"):
        self.kind = kind
        lib = _load(PORT_LIB if kind == "port" else REF_LIB_2D)
        p = "or2d_" if kind == "port" else "ref2d_"
        b = lambda n, r, a: _bind(lib, p + n, r, a)
        self._create = b("create", _vp, [_c_int, _c_int, _c_int] + [_c_double] * 4 + [_c_int])
        self._destroy = b("destroy", None, [_vp])
        self._dims = b("dims", None, [_vp, ctypes.POINTER(_c_int), ctypes.POINTER(_c_int)])
        self._set_q = b("set_q", None, [_vp, _dp])
        self._get_q = b("get_q", None, [_vp, _dp])
        self._init_problem = b("init_problem", None, [_vp, _c_int, _c_double, _c_double])
        self._get_masks = b("get_masks", None, [_vp, ctypes.POINTER(ctypes.c_uint8)])
        self._set_masks = b("set_masks", None, [_vp, ctypes.POINTER(ctypes.c_uint8)])
        self._get_levels = b("get_levels", None, [_vp, ctypes.POINTER(ctypes.c_int)])
        self._set_levels = b("set_levels", None, [_vp, ctypes.POINTER(ctypes.c_int)])
        self._prepare = b("prepare", None, [_vp, _c_double])
        self._fwt = b("fwt", None, [_vp, _c_double])
        self._iwt = b("iwt", None, [_vp, _c_int])
        self._interpolate = b("interpolate", None, [_vp, _c_int, _c_int])
        self._interpolate_all = b("interpolate_all", None, [_vp, _c_int])
        self._set_scalar = b("set_scalar", None, [_vp, _c_int])
        self._scalar_set_q = b("scalar_set_q", None, [_vp, _dp])
        self._scalar_get_q = b("scalar_get_q", None, [_vp, _dp])
        self._scalar_step = b("scalar_step", None, [_vp, _c_double, _c_double, _dp])
        self._manager = b("manager", None, [_vp, _c_int, _c_int, _c_int])
        self._apply_bc = b("apply_bc", None, [_vp, _c_double])
        self._set_bc_field = b("set_bc_field", None, [_vp, ctypes.POINTER(_c_int)])
        self._wt_call = b("wt_call", None, [_vp, _c_int, _c_int])
        self._step = b("step", None, [_vp] + [_c_double] * 5 + [_dp, _dp])
        self._set_freeze = b("set_freeze", None, [_vp, _c_int])
        if kind == "port":
            self._set_wenoz = b("set_wenoz", None, [_vp, _c_double, _c_double])
        else:
            self._set_wenoz_eps = b("set_wenoz_eps", None, [_vp, _c_double])
        self._run = b("run", _c_int, [_vp, _c_double, _c_double, _c_double, _c_int, _dp])
        self._threads = b("threads", _c_int, [])
        self.h = self._create(num_levels, nx_coarse, ny_coarse, x_min, x_max, y_min, y_max, bc_kind)
        nx, ny = _c_int(), _c_int()
        self._dims(self.h, ctypes.byref(nx), ctypes.byref(ny))
        self.nx, self.ny = nx.value, ny.value

    def __del__(self):
        if getattr(self, "h", None):
            self._destroy(self.h)
            self.h = None

    @property
    def threads(self):
        return self._threads()

    def set_q(self, q):
        q = np.ascontiguousarray(q, dtype=np.float64).reshape(self.ny + 6, self.nx + 6, 4)
        self._set_q(self.h, _ptr(q, ctypes.c_double))

    def get_q(self):
        q = np.empty((self.ny + 6, self.nx + 6, 4), np.float64)
        self._get_q(self.h, _ptr(q, ctypes.c_double))
        return q

    def init_problem(self, kind, a, b):
        self._init_problem(self.h, kind, a, b)

    def get_masks(self):
        m = np.empty((5, self.ny + 6, self.nx + 6), np.uint8)
        self._get_masks(self.h, _ptr(m, ctypes.c_uint8))
        return m

    def set_masks(self, m):
        m = np.ascontiguousarray(m, dtype=np.uint8).reshape(5, self.ny + 6, self.nx + 6)
        self._set_masks(self.h, _ptr(m, ctypes.c_uint8))

    def get_levels(self):
        lv = np.empty((4, self.ny, self.nx), np.int32)
        self._get_levels(self.h, _ptr(lv, ctypes.c_int))
        return lv

    def set_levels(self, lv):
        lv = np.ascontiguousarray(lv, dtype=np.int32).reshape(4, self.ny, self.nx)
        self._set_levels(self.h, _ptr(lv, ctypes.c_int))

    def prepare(self, tol):
        self._prepare(self.h, tol)

    def fwt(self, tol):
        self._fwt(self.h, tol)

    def iwt(self, mask_id=3):
        self._iwt(self.h, mask_id)

    def interpolate(self, from_id=4, to_id=3):
        self._interpolate(self.h, from_id, to_id)

    # scalar AWCM (Wavelet/main_2d_advect.cpp) ------------------------------------------------
    def set_scalar(self):
        """Switches the instance to the scalar advection path (field (Ny+6, Nx+6))."""
        self._set_scalar(self.h, 1)

    def scalar_set_q(self, q):
        q = np.ascontiguousarray(q, dtype=np.float64).reshape(self.ny + 6, self.nx + 6)
        self._scalar_set_q(self.h, _ptr(q, ctypes.c_double))

    def scalar_get_q(self):
        q = np.empty((self.ny + 6, self.nx + 6), np.float64)
        self._scalar_get_q(self.h, _ptr(q, ctypes.c_double))
        return q

    def scalar_step(self, tol, dt):
        out = np.zeros(4)
        self._scalar_step(self.h, tol, dt, _ptr(out, ctypes.c_double))
        return out

    def interpolate_all(self, from_id=0):
        """InterpolateAllGridEuler: the dense field from the points of mask `from_id`."""
        self._interpolate_all(self.h, from_id)

    def manager(self, op, mask_id, level_id=0):
        self._manager(self.h, op, mask_id, level_id)

    def apply_bc(self, t=0.0):
        self._apply_bc(self.h, t)

    def wt_call(self, which: int, mask_id: int = 0):
        """BOUNDARY_MANAGER_WT on the conserved field: 0 SetBottomBoundaryCondition(true, false),
        1 SetBottomBoundaryCondition(false, true), 2 BandingMask(mask mask_id)."""
        self._wt_call(self.h, which, mask_id)

    def set_bc_field(self, bc):
        """Attaches BOUNDARY_MANAGER_2D<TT> with the BOUNDARY_CONDITION field bc ((Ny+6, Nx+6) ints)."""
        bc = np.ascontiguousarray(bc, dtype=np.int32).reshape(self.ny + 6, self.nx + 6)
        self._set_bc_field(self.h, _ptr(bc, ctypes.c_int))

    def set_freeze(self, mode: int):
        """0 normal; 1 frozen mask (no PrepareEuler, no residue removal), LF speeds computed and
        recorded into the alpha buffer given to step(); 2 frozen mask with the LF speeds replayed."""
        self._set_freeze(self.h, int(mode))

    def set_wenoz(self, eps: float, tau_delta: float = 0.0):
        """WENO-Z epsilon of the face reconstructions (WENOZ5::eps, a public member of the
        reference solver, 1e-40 by default) and, for the restatement only, the smoothing
        tau = sqrt((b0-b2)^2 + tau_delta^2) of the differentiable mode (the reference has |.|)."""
        if self.kind == "port":
            self._set_wenoz(self.h, float(eps), float(tau_delta))
        else:
            if tau_delta != 0.0:
                raise ValueError("the reference's WENO-Z has no smoothed |b0 - b2|")
            self._set_wenoz_eps(self.h, float(eps))

    def step(self, tol, cfl, t, t_next, dt_fixed=0.0, alpha=None):
        out = np.zeros(8)
        ap = None if alpha is None else _ptr(alpha, ctypes.c_double)
        self._step(self.h, tol, cfl, t, t_next, dt_fixed, ap, _ptr(out, ctypes.c_double))
        return out

    def run(self, tol, cfl, t_end, max_steps=1 << 30):
        out = np.zeros(2)
        n = self._run(self.h, tol, cfl, t_end, max_steps, _ptr(out, ctypes.c_double))
        return n, out[0], out[1]


def run_tube(tube: dict, tol: float, cfl: float, t_end: float, scheme: int = 0, kind: str = "port"):
    """One 1D Riemann tube (a dict with num_levels, nx_coarse, x_min, x_max, x_interface, left,
    right) run from its initial state to t_end.  Returns (steps, t, sum |mask0|, q, masks, levels).
    A module-level function so that a process pool can run tubes side by side."""
    o = Oracle1D(tube["num_levels"], tube["nx_coarse"], tube["x_min"], tube["x_max"], scheme=scheme, kind=kind)
    o.init_riemann(tube["x_interface"], tube["left"], tube["right"])
    n, t, upd = o.run(tol, cfl, t_end)
    return n, t, upd, o.get_q(), o.get_masks(), o.get_levels()


def euler_flux(q, dim: int, direction: int = 0, gamma: float = 1.4, kind: str = "port"):
    """EULER_EQUATION_1D::ComputeFu (dim 1, q of shape (n, 3)) or EULER_EQUATION_2D::ComputeFu /
    ComputeGu (dim 2, direction 0 / 1, q of shape (n, 4)) of every state, by the restatement or by
    the reference's own class."""
    nc = 3 if dim == 1 else 4
    q = np.ascontiguousarray(q, dtype=np.float64).reshape(-1, nc)
    f = np.empty_like(q)
    if kind == "port":
        lib, name = _load(PORT_LIB), "or_euler%dd_flux" % dim
    else:
        lib, name = _load(REF_LIB_1D if dim == 1 else REF_LIB_2D), "ref_euler%dd_flux" % dim
    fn = getattr(lib, name)
    fn.restype = None
    if dim == 1:
        fn.argtypes = [_dp, _dp, _c_int, _c_double]
        fn(_ptr(q, ctypes.c_double), _ptr(f, ctypes.c_double), q.shape[0], gamma)
    else:
        fn.argtypes = [_dp, _dp, _c_int, _c_int, _c_double]
        fn(_ptr(q, ctypes.c_double), _ptr(f, ctypes.c_double), q.shape[0], direction, gamma)
    return f


def euler_spectral_radius(q, dim: int, direction: int = 0, gamma: float = 1.4, kind: str = "port"):
    """EULER_EQUATION_1D::Spectral_Radius or EULER_EQUATION_2D::Spectral_RadiusX / Y of every state."""
    nc = 3 if dim == 1 else 4
    q = np.ascontiguousarray(q, dtype=np.float64).reshape(-1, nc)
    out = np.empty(q.shape[0])
    if kind == "port":
        lib, name = _load(PORT_LIB), "or_euler%dd_sr" % dim
    else:
        lib, name = _load(REF_LIB_1D if dim == 1 else REF_LIB_2D), "ref_euler%dd_sr" % dim
    fn = getattr(lib, name)
    fn.restype = None
    if dim == 1:
        fn.argtypes = [_dp, _dp, _c_int, _c_double]
        fn(_ptr(q, ctypes.c_double), _ptr(out, ctypes.c_double), q.shape[0], gamma)
    else:
        fn.argtypes = [_dp, _dp, _c_int, _c_int, _c_double]
        fn(_ptr(q, ctypes.c_double), _ptr(out, ctypes.c_double), q.shape[0], direction, gamma)
    return out
