"""Host-side solver objects over the C-ABI.

``AWCM2D`` is one 2D instance (AWCM_2D + its field, stage copies and boundary manager);
``AWCM1DBatch`` is a batch of independent 1D instances advanced by one persistent launch per RK3
step; ``AWCM1D`` is a batch of one.  Method names and argument meanings follow the checker in
``oracle/`` so the parity tests read the same against both.

Host layouts (reference layout, ghost ring of 3):
  1D state (Nx+6, 3) float64; 2D state (Ny+6, Nx+6, 4) float64;
  masks (5, ...) uint8 planes mask_temp, mask0..mask3; levels (4, ...) int32 planes.
"""
from __future__ import annotations

import ctypes

import numpy as np

from ._lib import AWCM_OK, AwcmError, P_double, P_int, P_u8, c_void_p, call, load, ptr

ERR_NONFINITE = 5

AAZ, CR, APD, CL, RR, BAND = 0, 1, 2, 3, 4, 5
BC_TRANSMISSIVE, BC_DOUBLE_MACH, BC_PERIODIC, BC_SHOCK_VORTEX, BC_GENERIC, BC_WIND_TUNNEL = 0, 1, 2, 3, 4, 5
# BOUNDARY_CONDITION values of the generic managers (BOUNDARY_MANAGER_2D.h:7-13)
SOLID_WALL, PERIODIC, EXTRAPOLATION_ZERO_ORDER, SPECIFIED, FLUID = -4, -3, -2, -1, 0
PROBLEM_QUADRANTS, PROBLEM_DOUBLE_MACH, PROBLEM_VORTEX, PROBLEM_SHOCK_VORTEX, PROBLEM_WIND_TUNNEL = 0, 1, 2, 3, 4
WENOZ, WENO5 = 0, 1
# 1D scalar AWCM (the path of Wavelet/main_1d_advect.cpp): a batch scheme like the two above.
SCALAR_ADVECTION = 2


def euler_flux(q_dev, f_dev, n: int, dim: int, direction: int = 0, gamma: float = 1.4, stream=None):
    """EULER_EQUATION_1D::ComputeFu (dim 1) or EULER_EQUATION_2D::ComputeFu / ComputeGu (dim 2,
    direction 0 / 1) on n device-resident states; q_dev, f_dev are device addresses (ints)."""
    if dim == 1:
        call("euler1d_flux", q_dev, f_dev, n, gamma, stream)
    else:
        call("euler2d_flux", q_dev, f_dev, n, direction, gamma, stream)


def euler_spectral_radius(q_dev, s_dev, n: int, dim: int, direction: int = 0, gamma: float = 1.4, stream=None):
    """EULER_EQUATION_1D::Spectral_Radius or EULER_EQUATION_2D::Spectral_RadiusX / Y on n
    device-resident states."""
    if dim == 1:
        call("euler1d_spectral_radius", q_dev, s_dev, n, gamma, stream)
    else:
        call("euler2d_spectral_radius", q_dev, s_dev, n, direction, gamma, stream)


def measure_fp64_peak(iters: int = 20000, repeats: int = 5) -> float:
    """Dense FP64 FMA throughput of the current device, TFLOP/s."""
    v = ctypes.c_double()
    call("awcm_measure_fp64_peak", iters, repeats, ctypes.byref(v))
    return v.value


class AWCM2D:
    """One 2D AWCM compressible-Euler instance resident on the GPU."""

    def __init__(self, num_levels: int, nx_coarse: int, ny_coarse: int, x_min: float, x_max: float,
                 y_min: float, y_max: float, bc_kind: int = BC_TRANSMISSIVE):
        h = c_void_p()
        call("awcm2d_create", num_levels, nx_coarse, ny_coarse, x_min, x_max, y_min, y_max, bc_kind,
             ctypes.byref(h))
        self.h = h
        nx, ny = ctypes.c_int(), ctypes.c_int()
        call("awcm2d_dims", self.h, ctypes.byref(nx), ctypes.byref(ny))
        self.nx, self.ny = nx.value, ny.value
        self.num_levels = num_levels

    def close(self):
        if getattr(self, "h", None) is not None and self.h.value:
            call("awcm2d_destroy", self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # state ------------------------------------------------------------------------------------
    def set_q(self, q):
        q = np.ascontiguousarray(q, dtype=np.float64).reshape(self.ny + 6, self.nx + 6, 4)
        call("awcm2d_set_q", self.h, ptr(q, ctypes.c_double))

    def get_q(self):
        q = np.empty((self.ny + 6, self.nx + 6, 4), np.float64)
        call("awcm2d_get_q", self.h, ptr(q, ctypes.c_double))
        return q

    def get_masks(self):
        m = np.empty((5, self.ny + 6, self.nx + 6), np.uint8)
        call("awcm2d_get_masks", self.h, ptr(m, ctypes.c_uint8))
        return m

    def set_masks(self, m):
        m = np.ascontiguousarray(m, dtype=np.uint8).reshape(5, self.ny + 6, self.nx + 6)
        call("awcm2d_set_masks", self.h, ptr(m, ctypes.c_uint8))

    def get_levels(self):
        lv = np.empty((4, self.ny, self.nx), np.int32)
        call("awcm2d_get_levels", self.h, ptr(lv, ctypes.c_int))
        return lv

    def set_levels(self, lv):
        lv = np.ascontiguousarray(lv, dtype=np.int32).reshape(4, self.ny, self.nx)
        call("awcm2d_set_levels", self.h, ptr(lv, ctypes.c_int))

    def init_problem(self, kind, a, b):
        call("awcm2d_init_problem", self.h, kind, a, b)

    # passes -----------------------------------------------------------------------------------
    def prepare(self, tol):
        call("awcm2d_prepare", self.h, tol)

    def fwt(self, tol):
        call("awcm2d_fwt", self.h, tol)

    def iwt(self, mask_id=3):
        call("awcm2d_iwt", self.h, mask_id)

    def interpolate_all(self, from_id=0):
        """InterpolateAllGridEuler: interpolate all four components at every grid point outside
        mask `from_id` (the dense field)."""
        call("awcm2d_interpolate_all", self.h, from_id)

    def interpolate(self, from_id=4, to_id=3):
        call("awcm2d_interpolate", self.h, from_id, to_id)

    def manager(self, op, mask_id, level_id=0):
        call("awcm2d_manager", self.h, op, mask_id, level_id)

    def apply_bc(self, t=0.0):
        call("awcm2d_apply_bc", self.h, t)

    def wt_set_bottom(self, x_direction: bool, y_direction: bool):
        """BOUNDARY_MANAGER_WT::SetBottomBoundaryCondition(x_direction, y_direction)."""
        call("awcm2d_wt_set_bottom", self.h, int(x_direction), int(y_direction))

    def set_bc_field(self, bc):
        """Attaches the enum-driven BOUNDARY_MANAGER_2D: bc is (Ny+6, Nx+6) BOUNDARY_CONDITION values."""
        bc = np.ascontiguousarray(bc, dtype=np.int32).reshape(self.ny + 6, self.nx + 6)
        call("awcm2d_set_bc_field", self.h, ptr(bc, ctypes.c_int))

    # stepping ---------------------------------------------------------------------------------
    def step(self, tol, cfl, t, t_next, dt_fixed=0.0):
        out = np.zeros(8)
        call("awcm2d_step", self.h, tol, cfl, t, t_next, dt_fixed, ptr(out, ctypes.c_double))
        return out

    def advance(self, tol, cfl, t_start, t_end, n_steps):
        """n_steps graph replays without host round trips; returns (t, steps, sum|mask0|, stage points)."""
        out = np.zeros(4)
        call("awcm2d_advance", self.h, tol, cfl, t_start, t_end, n_steps, ptr(out, ctypes.c_double))
        return out[0], int(out[1]), out[2], out[3]

    def run(self, tol, cfl, t_end, max_steps=1 << 30, chunk=64):
        t, steps, upd = 0.0, 0, 0.0
        while steps < max_steps and t < t_end:
            n = min(chunk, max_steps - steps)
            t, k, u, _ = self.advance(tol, cfl, t, t_end, n)
            steps += k
            upd += u
            if k < n:
                break
        return steps, t, upd

    def profile_step(self, tol, cfl, t, t_end):
        """One eagerly launched step with phase events; returns a dict of device times and counts."""
        out = np.zeros(19)
        call("awcm2d_profile_step", self.h, tol, cfl, t, t_end, ptr(out, ctypes.c_double))
        return {
            "prepare_ms": out[0], "setup_ms": out[1], "face_ms": out[2:5].tolist(),
            "update_ms": out[5:8].tolist(), "between_ms": out[8], "post_ms": out[9], "total_ms": out[10],
            "faces": out[11:14].tolist(), "stage_points": out[14:17].tolist(), "mask0": out[17], "dt": out[18],
        }

    def profile_kernels(self, tol, cfl, t, t_end, cap=512):
        """One step with an event after every kernel; returns [(kernel, ms)] in launch order."""
        names = ctypes.create_string_buffer(32 * cap)
        ms = np.zeros(cap)
        n = ctypes.c_int()
        call("awcm2d_profile_kernels", self.h, tol, cfl, t, t_end, cap, names, ptr(ms, ctypes.c_double), ctypes.byref(n))
        raw = names.raw
        return [(raw[32 * k:32 * k + 32].split(b"\0")[0].decode(), float(ms[k])) for k in range(n.value)]

    def set_prepare_mode(self, mode: int):
        """0: persistent cooperative prepare kernel; 1: one launch per pass (the default)."""
        call("awcm2d_set_prepare_mode", self.h, mode)

    def set_spin_limit(self, polls: int):
        """Test hook: polls before a grid-barrier wait of the persistent prepare gives up (0 = default)."""
        call("awcm2d_set_spin_limit", self.h, int(polls))

    def launches_per_step(self):
        n = ctypes.c_int()
        call("awcm2d_launches_per_step", self.h, ctypes.byref(n))
        return n.value

    @property
    def stream(self) -> int:
        s = c_void_p()
        call("awcm2d_stream", self.h, ctypes.byref(s))
        return s.value or 0

    # state file -------------------------------------------------------------------------------
    def geometry(self):
        """(num_levels, nx_coarse, ny_coarse, bc_kind, x_min, x_max, y_min, y_max, gamma)."""
        class _G(ctypes.Structure):
            _fields_ = [("num_levels", ctypes.c_int), ("nx_coarse", ctypes.c_int), ("ny_coarse", ctypes.c_int),
                        ("bc_kind", ctypes.c_int), ("x_min", ctypes.c_double), ("x_max", ctypes.c_double),
                        ("y_min", ctypes.c_double), ("y_max", ctypes.c_double), ("gamma", ctypes.c_double)]
        gm = _G()
        call("awcm2d_get_geometry", self.h, ctypes.byref(gm))
        return (gm.num_levels, gm.nx_coarse, gm.ny_coarse, gm.bc_kind, gm.x_min, gm.x_max, gm.y_min, gm.y_max,
                gm.gamma)

    def save_state(self, path, t=0.0, step=0):
        """Binary state file: masks, levels and the state on mask0 (awcm2d_save_state)."""
        call("awcm2d_save_state", self.h, str(path).encode(), float(t), int(step))

    def load_state(self, path):
        """Restores state, masks and levels from a state file; returns (t, step)."""
        t, step = ctypes.c_double(), ctypes.c_longlong()
        call("awcm2d_load_state", self.h, str(path).encode(), ctypes.byref(t), ctypes.byref(step))
        return t.value, step.value

    # frozen-mask run and adjoint --------------------------------------------------------------
    @property
    def tape_stride(self) -> int:
        """Doubles of LF-speed tape per step: 3 stages x (alpha_x[Ny], alpha_y[Nx])."""
        return 3 * (self.nx + self.ny)

    def frozen_run(self, t0, dt, n_steps, replay=False):
        """n_steps frozen-mask steps (no PrepareEuler / residue removal, fixed dt); LF speeds
        recorded on the tape, or replayed from it.  Returns (t, device ms, sum |mask0|)."""
        out = np.zeros(3)
        call("awcm2d_frozen_run", self.h, t0, dt, n_steps, 2 if replay else 1, ptr(out, ctypes.c_double))
        return out[0], out[1], out[2]

    def set_wenoz(self, eps: float, tau_delta: float = 0.0):
        """WENO-Z epsilon of the face reconstructions (WENOZ5::eps; 1e-40 as in the reference) and
        the smoothing tau = sqrt((b0-b2)^2 + tau_delta^2) (0: |b0 - b2| as in the reference).
        The gradient checks run the differentiable mode eps = tau_delta = 1e-6."""
        call("awcm2d_set_wenoz", self.h, float(eps), float(tau_delta))

    def adjoint(self, t0, dt, n_steps, target, checkpoint_every=0, replay=False, with_grad=True):
        """Loss 1/2 |rho(t0 + n dt) - target|^2 of the frozen run from the current state and its
        gradient w.r.t. the state at t0 ((Ny+6, Nx+6, 4), zero on ghosts).  Returns
        (loss, grad or None, info dict)."""
        tgt = np.ascontiguousarray(target, dtype=np.float64).reshape(self.ny, self.nx)
        grad = np.empty((self.ny + 6, self.nx + 6, 4), np.float64) if with_grad else None
        out = np.zeros(5)
        call("awcm2d_adjoint", self.h, t0, dt, n_steps, checkpoint_every, 2 if replay else 1,
             ptr(tgt, ctypes.c_double), ptr(grad, ctypes.c_double) if with_grad else None,
             ptr(out, ctypes.c_double))
        info = {"forward_ms": out[1], "reverse_ms": out[2], "checkpoint_every": int(out[3]), "device_bytes": out[4]}
        return out[0], grad, info

    def get_alpha_tape(self, n_steps):
        t = np.empty((n_steps, self.tape_stride), np.float64)
        call("awcm2d_get_alpha_tape", self.h, n_steps, ptr(t, ctypes.c_double))
        return t

    def set_alpha_tape(self, tape):
        t = np.ascontiguousarray(tape, dtype=np.float64).reshape(-1, self.tape_stride)
        call("awcm2d_set_alpha_tape", self.h, t.shape[0], ptr(t, ctypes.c_double))


class AWCM2DScalar:
    """Scalar AWCM instance (the path of Wavelet/main_2d_advect.cpp): one field advected with unit
    velocity, periodic; masks and levels as for AWCM2D."""

    def __init__(self, num_levels: int, nx_coarse: int, ny_coarse: int, x_min: float, x_max: float,
                 y_min: float, y_max: float):
        h = c_void_p()
        call("awcm2d_create_scalar", num_levels, nx_coarse, ny_coarse, x_min, x_max, y_min, y_max, ctypes.byref(h))
        self.h = h
        nx, ny = ctypes.c_int(), ctypes.c_int()
        call("awcm2d_dims", self.h, ctypes.byref(nx), ctypes.byref(ny))
        self.nx, self.ny = nx.value, ny.value

    def close(self):
        if getattr(self, "h", None) is not None and self.h.value:
            call("awcm2d_destroy", self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_q(self, q):
        q = np.ascontiguousarray(q, dtype=np.float64).reshape(self.ny + 6, self.nx + 6)
        call("awcm2d_scalar_set_q", self.h, ptr(q, ctypes.c_double))

    def get_q(self):
        q = np.empty((self.ny + 6, self.nx + 6), np.float64)
        call("awcm2d_scalar_get_q", self.h, ptr(q, ctypes.c_double))
        return q

    def get_masks(self):
        m = np.empty((5, self.ny + 6, self.nx + 6), np.uint8)
        call("awcm2d_get_masks", self.h, ptr(m, ctypes.c_uint8))
        return m

    def get_levels(self):
        lv = np.empty((4, self.ny, self.nx), np.int32)
        call("awcm2d_get_levels", self.h, ptr(lv, ctypes.c_int))
        return lv

    def advance(self, tol, dt, t, n_steps):
        """n_steps driver passes at the fixed dt; returns (t, steps, sum |mask0|)."""
        out = np.zeros(3)
        call("awcm2d_scalar_advance", self.h, tol, dt, t, n_steps, ptr(out, ctypes.c_double))
        return out[0], int(out[1]), out[2]

    @property
    def stream(self) -> int:
        s = c_void_p()
        call("awcm2d_stream", self.h, ctypes.byref(s))
        return s.value or 0


class AWCM1DBatch:
    """Independent 1D AWCM instances advanced together (one persistent launch per RK3 step)."""

    def __init__(self, num_levels, nx_coarse, x_min, x_max, gamma: float = 1.4, scheme: int = WENOZ):
        num_levels = np.ascontiguousarray(num_levels, dtype=np.int32)
        n = len(num_levels)
        nxc = np.ascontiguousarray(np.broadcast_to(nx_coarse, (n,)), dtype=np.int32)
        xmin = np.ascontiguousarray(np.broadcast_to(x_min, (n,)), dtype=np.float64)
        xmax = np.ascontiguousarray(np.broadcast_to(x_max, (n,)), dtype=np.float64)
        h = c_void_p()
        call("awcm1d_batch_create", n, ptr(num_levels, ctypes.c_int), ptr(nxc, ctypes.c_int),
             ptr(xmin, ctypes.c_double), ptr(xmax, ctypes.c_double), gamma, scheme, ctypes.byref(h))
        self.h = h
        self.n = n
        self.nx = []
        for k in range(n):
            v = ctypes.c_int()
            call("awcm1d_batch_nx", self.h, k, ctypes.byref(v))
            self.nx.append(v.value)

    def close(self):
        if getattr(self, "h", None) is not None and self.h.value:
            call("awcm1d_batch_destroy", self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_q(self, k, q):
        q = np.ascontiguousarray(q, dtype=np.float64).reshape(self.nx[k] + 6, 3)
        call("awcm1d_batch_set_q", self.h, k, ptr(q, ctypes.c_double))

    def get_q(self, k):
        q = np.empty((self.nx[k] + 6, 3), np.float64)
        call("awcm1d_batch_get_q", self.h, k, ptr(q, ctypes.c_double))
        return q

    def get_masks(self, k):
        m = np.empty((5, self.nx[k] + 6), np.uint8)
        call("awcm1d_batch_get_masks", self.h, k, ptr(m, ctypes.c_uint8))
        return m

    def set_masks(self, k, m):
        m = np.ascontiguousarray(m, dtype=np.uint8).reshape(5, self.nx[k] + 6)
        call("awcm1d_batch_set_masks", self.h, k, ptr(m, ctypes.c_uint8))

    def get_levels(self, k):
        lv = np.empty((4, self.nx[k]), np.int32)
        call("awcm1d_batch_get_levels", self.h, k, ptr(lv, ctypes.c_int))
        return lv

    def set_levels(self, k, lv):
        lv = np.ascontiguousarray(lv, dtype=np.int32).reshape(4, self.nx[k])
        call("awcm1d_batch_set_levels", self.h, k, ptr(lv, ctypes.c_int))

    def init_riemann(self, k, x_interface, left, right):
        l = np.ascontiguousarray(left, dtype=np.float64)
        r = np.ascontiguousarray(right, dtype=np.float64)
        call("awcm1d_batch_init_riemann", self.h, k, x_interface, ptr(l, ctypes.c_double), ptr(r, ctypes.c_double))

    def set_run(self, tol, cfl, t, t_end, dt_fixed=0.0):
        f = lambda v: np.ascontiguousarray(np.broadcast_to(v, (self.n,)), dtype=np.float64)
        a, b, c, d = f(tol), f(cfl), f(t), f(t_end)
        call("awcm1d_batch_set_run", self.h, ptr(a, ctypes.c_double), ptr(b, ctypes.c_double),
             ptr(c, ctypes.c_double), ptr(d, ctypes.c_double), dt_fixed)

    def steps(self, n_steps: int):
        call("awcm1d_batch_steps", self.h, n_steps)

    def run_all(self, max_steps: int = (1 << 31) - 1):
        """Every unfinished instance to its end time (at most max_steps steps each) in one launch,
        each instance's steps back to back on one CTA (asynchronous, like steps)."""
        call("awcm1d_batch_run", self.h, max_steps)

    def sync(self):
        call("awcm1d_batch_sync", self.h)

    def status(self, k):
        """out[16] of instance k (awcm1d_batch_status); out[14] = 5 marks a non-finite state,
        which is returned here rather than raised (check_finite raises it)."""
        out = np.zeros(16)
        rc = load().awcm1d_batch_status(self.h, k, ptr(out, ctypes.c_double))
        if rc not in (AWCM_OK, ERR_NONFINITE):
            raise AwcmError("awcm1d_batch_status", rc, load().awcm_last_error().decode(errors="replace"))
        return out

    def check_finite(self, k):
        """Raises AwcmError(ERR_NONFINITE) if instance k stopped on a NaN or infinite wave speed."""
        call("awcm1d_batch_status", self.h, k, ptr(np.zeros(16), ctypes.c_double))

    def totals(self):
        out = np.zeros(3)
        call("awcm1d_batch_totals", self.h, ptr(out, ctypes.c_double))
        return out

    def pass_(self, k, op, mask_id, level_id=0):
        call("awcm1d_batch_pass", self.h, k, op, mask_id, level_id)

    def set_launch(self, threads: int, ctas_per_sm: int = 0):
        call("awcm1d_batch_set_launch", self.h, threads, ctas_per_sm)

    @property
    def stream(self) -> int:
        s = c_void_p()
        call("awcm1d_batch_stream", self.h, ctypes.byref(s))
        return s.value or 0


class AWCM1DScalar:
    """Scalar 1D AWCM instances (the path of Wavelet/main_1d_advect.cpp:48-224): one field advected
    with unit speed at a fixed dt, batched like the Euler instances (scheme SCALAR_ADVECTION)."""

    def __init__(self, num_levels, nx_coarse, x_min, x_max):
        self.b = AWCM1DBatch(num_levels, nx_coarse, x_min, x_max, 1.4, SCALAR_ADVECTION)
        self.n, self.nx = self.b.n, self.b.nx
        self._t = np.zeros(self.n)

    def set_q(self, k, q):
        """q: the field at the Nx + 6 points -3 .. Nx+2 (ghosts included)."""
        q = np.ascontiguousarray(q, dtype=np.float64).reshape(self.nx[k] + 6)
        full = np.zeros((self.nx[k] + 6, 3))
        full[:, 0] = q
        self.b.set_q(k, full)

    def get_q(self, k):
        return np.ascontiguousarray(self.b.get_q(k)[:, 0])

    def get_masks(self, k):
        return self.b.get_masks(k)

    def get_levels(self, k):
        return self.b.get_levels(k)

    def advance(self, tol, dt: float, n_steps: int):
        """n_steps driver passes of every instance at the fixed dt (one dt for the batch: the
        driver's 0.5 dx is the caller's choice); returns the per-instance time."""
        self.b.set_run(tol, 0.0, self._t, np.inf, float(dt))
        self.b.steps(n_steps)
        self.b.sync()
        self._t = np.array([self.b.status(k)[0] for k in range(self.n)])
        return self._t.copy()

    def status(self, k):
        return self.b.status(k)

    def totals(self):
        return self.b.totals()


class AWCM1D:
    """A single 1D instance with the checker's call shape (a batch of one)."""

    def __init__(self, num_levels: int, nx_coarse: int, x_min: float, x_max: float, gamma: float = 1.4,
                 scheme: int = WENOZ):
        self.b = AWCM1DBatch([num_levels], nx_coarse, x_min, x_max, gamma, scheme)
        self.nx = self.b.nx[0]

    def set_q(self, q):
        self.b.set_q(0, q)

    def get_q(self):
        return self.b.get_q(0)

    def get_masks(self):
        return self.b.get_masks(0)

    def set_masks(self, m):
        self.b.set_masks(0, m)

    def get_levels(self):
        return self.b.get_levels(0)

    def set_levels(self, lv):
        self.b.set_levels(0, lv)

    def init_riemann(self, x_interface, left, right):
        self.b.init_riemann(0, x_interface, left, right)

    def prepare(self, tol):
        """AWCM_1D::PrepareEuler(Q, tol)."""
        call("awcm1d_batch_prepare", self.b.h, 0, tol)

    def fwt(self, tol):
        """WAVELET_1D::ForwardWaveletTransformEuler(Q, mra, mask0, tol)."""
        call("awcm1d_batch_fwt", self.b.h, 0, tol)

    def iwt(self, mask_id=3):
        """WAVELET_1D::InverseWaveletTransformEuler(Q, mra, mask)."""
        call("awcm1d_batch_iwt", self.b.h, 0, mask_id)

    def interpolate(self, from_id=4, to_id=3):
        """WAVELET_1D::InterpolateEuler(Q, mra, mask_from, mask_to)."""
        call("awcm1d_batch_interpolate", self.b.h, 0, from_id, to_id)

    def manager(self, op, mask_id, level_id=0):
        """AWCM_MANAGER_1D pass `op` (AAZ, CR, APD, CL, RR, BAND) on mask `mask_id`."""
        call("awcm1d_batch_manager", self.b.h, 0, op, mask_id, level_id)

    def apply_bc(self):
        """The instance's ghost fill (transmissive BOUNDARY_MANAGER, or the attached generic one)."""
        call("awcm1d_batch_apply_bc", self.b.h, 0)

    def set_bc_field(self, bc):
        """Attaches the enum-driven BOUNDARY_MANAGER_1D: bc is Nx+6 BOUNDARY_CONDITION values."""
        bc = np.ascontiguousarray(bc, dtype=np.int32).reshape(self.nx + 6)
        call("awcm1d_batch_set_bc_field", self.b.h, 0, ptr(bc, ctypes.c_int))

    def step(self, tol, cfl, t, t_next):
        """One driver-loop pass; returns the checker's out[10] (dt, do_print, |mask0..3|, alphas, speed)."""
        self.b.set_run(tol, cfl, t, t_next)
        self.b.steps(1)
        self.b.check_finite(0)
        s = self.b.status(0)
        out = np.zeros(10)
        out[0], out[1] = s[1], s[2]
        out[2:6] = s[5:9]
        out[6:9] = s[10:13]
        out[9] = s[9]
        return out

    def run(self, tol, cfl, t_end, max_steps=1 << 30):
        """The driver loop from t = 0 to t_end (at most max_steps steps) as one launch, the instance
        staged into shared memory once; returns (steps, t, sum over the steps of |mask0|)."""
        self.b.set_run(tol, cfl, 0.0, t_end)
        self.b.run_all(min(max_steps, (1 << 31) - 1))
        s = self.b.status(0)
        return int(s[4]), s[0], s[13]
