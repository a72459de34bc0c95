"""Python binding of libccfv (the C ABI in include/ccfv.h).

Mirrors the reference's in-process interface of T2S4_Parareal.cu: a
``GPUContext`` holding the state ``v_d_Cn`` and the functions
``GpuOneStep`` / ``CoarsePropagator`` / ``FinePropagator`` with the same
argument meaning, plus a ``Solver`` object for the rest of the ABI.

Device memory and streams come from PyTorch (plumbing only); all compute runs
in libccfv's CUDA kernels.  Loading fails loudly when the library is missing:
there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

PKG_DIR = Path(__file__).resolve().parents[1]
# CCFV_LIBRARY selects another build of libccfv (same C ABI), e.g. for A/B timing.
LIB_PATH = Path(os.environ["CCFV_LIBRARY"]) if os.environ.get("CCFV_LIBRARY") else \
    PKG_DIR / "lib" / "libccfv.so"
HEADER = PKG_DIR.parent / "include" / "ccfv.h"

OK, ERR_INVALID, ERR_CUDA, ERR_NOMEM, ERR_UNSUPPORTED, ERR_HALO = 0, 1, 2, 3, 4, 5
ERR_BUDGET, ERR_NOT_FOUND, ERR_CANCELLED, ERR_TIMEOUT = 6, 7, 8, 9
BC_COMPAT, BC_PERIODIC = 0, 1
VEL_REF_ROT4, VEL_CONST, VEL_ROTATION, VEL_SWIRL = 0, 1, 2, 3
SCHEME_REFERENCE, SCHEME_CONSISTENT = 0, 1
SRC_NONE, SRC_GAUSSIAN = 0, 1
FP64, FP32 = 0, 1
MEM_DEVICE, MEM_HOST = 0, 1
FORM_STANDARD, FORM_DELTA = 0, 1
COARSE_THETA_AUTO = -1.0  # ccfv_parareal_opts::coarse_theta: damping rule
MAX_ITERS = 128


class CcfvError(RuntimeError):
    def __init__(self, status: int, msg: str = ""):
        self.status = status
        super().__init__(f"ccfv error {status}: {msg}")


class Grid(C.Structure):
    _fields_ = [
        ("nx", C.c_int), ("ny", C.c_int),
        ("x_min", C.c_double), ("x_max", C.c_double),
        ("y_min", C.c_double), ("y_max", C.c_double),
        ("bc", C.c_int), ("velocity", C.c_int),
        ("vel_params", C.c_double * 4),
        ("K", C.c_double),
        ("scheme", C.c_int),
        ("source", C.c_int),
        ("source_params", C.c_double * 5),
    ]


class PararealOpts(C.Structure):
    _fields_ = [
        ("t0", C.c_double), ("t1", C.c_double),
        ("nt_fine", C.c_int), ("n_slices", C.c_int), ("coarse_ratio", C.c_int),
        ("tol", C.c_double), ("kmax", C.c_int), ("coarse_precision", C.c_int),
        ("form", C.c_int), ("mem", C.c_int), ("d_ref", C.c_void_p),
        ("coarse_theta", C.c_double),
    ]


class Stats(C.Structure):
    _fields_ = [
        ("iterations", C.c_int), ("converged", C.c_int),
        ("update", C.c_double * MAX_ITERS),
        ("fine_cell_updates", C.c_double), ("coarse_cell_updates", C.c_double),
        ("ms", C.c_double), ("fine_ms", C.c_double), ("coarse_ms", C.c_double),
        ("fine_sweep_launches", C.c_longlong), ("fine_sweep_cells", C.c_longlong),
        ("err_max", C.c_double * MAX_ITERS), ("err_l2", C.c_double * MAX_ITERS),
    ]

    def as_dict(self) -> dict:
        n = self.iterations
        return dict(iterations=n, converged=bool(self.converged),
                    update=[self.update[i] for i in range(min(n, MAX_ITERS))],
                    fine_cell_updates=self.fine_cell_updates,
                    coarse_cell_updates=self.coarse_cell_updates, ms=self.ms,
                    fine_ms=self.fine_ms, coarse_ms=self.coarse_ms,
                    fine_sweep_launches=self.fine_sweep_launches,
                    fine_sweep_cells=self.fine_sweep_cells,
                    err_max=[self.err_max[i] for i in range(min(n, MAX_ITERS))],
                    err_l2=[self.err_l2[i] for i in range(min(n, MAX_ITERS))])


class Problem(C.Structure):
    _fields_ = [("grid", Grid), ("opts", PararealOpts), ("C0", C.c_void_p), ("C_T", C.c_void_p)]


class ServerOpts(C.Structure):
    _fields_ = [("device", C.c_int), ("hbm_budget_bytes", C.c_size_t), ("max_active", C.c_int)]


REQ_QUEUED, REQ_RUNNING, REQ_DONE, REQ_FAILED, REQ_CANCELLED = 0, 1, 2, 3, 4

_lib = None

# Every function declared in include/ccfv.h with its ctypes signature.
_SIGS = {
    "ccfv_create": (C.c_int, [C.POINTER(C.c_void_p), C.POINTER(Grid), C.c_int]),
    "ccfv_destroy": (C.c_int, [C.c_void_p]),
    "ccfv_strerror": (C.c_char_p, [C.c_int]),
    "ccfv_check": (C.c_int, [C.c_void_p, C.c_void_p]),
    "ccfv_step": (C.c_int, [C.c_void_p, C.c_void_p, C.c_double, C.c_double, C.c_void_p]),
    "ccfv_fine": (C.c_int, [C.c_void_p, C.c_void_p, C.c_double, C.c_double, C.c_int, C.c_void_p]),
    "ccfv_coarse": (C.c_int, [C.c_void_p, C.c_void_p, C.c_double, C.c_double, C.c_int, C.c_int,
                              C.c_void_p]),
    "ccfv_coarse_ex": (C.c_int, [C.c_void_p, C.c_void_p, C.c_double, C.c_double, C.c_int,
                                 C.c_int, C.c_double, C.c_void_p]),
    "ccfv_coarse_theta": (C.c_int, [C.POINTER(Grid), C.POINTER(PararealOpts),
                                    C.POINTER(C.c_double)]),
    "ccfv_run": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_double, C.c_double, C.c_int,
                           C.c_void_p]),
    "ccfv_parareal": (C.c_int, [C.c_void_p, C.POINTER(PararealOpts), C.c_void_p, C.c_void_p,
                                C.POINTER(Stats), C.c_void_p]),
    "ccfv_kernel_launches": (C.c_uint64, []),
    "ccfv_last_error": (C.c_char_p, [C.c_void_p]),
    "ccfv_exact_ref": (C.c_int, [C.c_void_p, C.c_void_p, C.c_double, C.c_void_p]),
    "ccfv_gaussians": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_int,
                                 C.c_void_p]),
    "ccfv_error_norms": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(C.c_double),
                                   C.POINTER(C.c_double), C.c_void_p]),
    "ccfv_batch_solve": (C.c_int, [C.c_int, C.POINTER(Problem), C.POINTER(Stats), C.c_int,
                                   C.c_void_p]),
    "ccfv_server_create": (C.c_int, [C.POINTER(C.c_void_p), C.POINTER(ServerOpts)]),
    "ccfv_server_submit": (C.c_int, [C.c_void_p, C.POINTER(Problem), C.POINTER(C.c_uint64)]),
    "ccfv_server_poll": (C.c_int, [C.c_void_p, C.c_uint64, C.POINTER(C.c_int), C.POINTER(Stats),
                                   C.POINTER(C.c_double)]),
    "ccfv_server_wait": (C.c_int, [C.c_void_p, C.c_uint64, C.c_double, C.POINTER(Stats),
                                   C.POINTER(C.c_double)]),
    "ccfv_server_cancel": (C.c_int, [C.c_void_p, C.c_uint64]),
    "ccfv_server_info": (C.c_int, [C.c_void_p, C.POINTER(C.c_size_t), C.POINTER(C.c_int),
                                   C.POINTER(C.c_int)]),
    "ccfv_server_destroy": (C.c_int, [C.c_void_p]),
    "ccfv_fine_slices": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_double, C.c_double,
                                   C.c_double, C.c_int, C.c_void_p]),
    "ccfv_correct": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p,
                               C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_double),
                               C.c_void_p]),
    "ccfv_autotune": (C.c_int, [C.c_void_p, C.c_double, C.c_int, C.POINTER(C.c_int), C.c_void_p]),
    "ccfv_sweep_plan": (C.c_int, [C.c_void_p, C.c_double, C.c_int, C.POINTER(C.c_int),
                                  C.POINTER(C.c_int)]),
    "ccfv_step_noalloc": (C.c_int, [C.POINTER(Grid), C.c_void_p, C.c_double, C.c_double,
                                    C.c_void_p]),
}


def lib():
    """Load libccfv.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(f"{LIB_PATH} is missing: build it with `make -C {PKG_DIR}` "
                               "(the CUDA path has no fallback)")
        L = C.CDLL(str(LIB_PATH))
        for name, (res, args) in _SIGS.items():
            fn = getattr(L, name)
            fn.restype, fn.argtypes = res, args
        _lib = L
    return _lib


def kernel_launches() -> int:
    return int(lib().ccfv_kernel_launches())


def make_grid(nx, ny=None, *, bc=BC_COMPAT, velocity=VEL_REF_ROT4, vel_params=(0, 0, 0, 0),
              K=0.0, domain=None, scheme=SCHEME_REFERENCE, source=SRC_NONE,
              source_params=(0, 0, 0, 1, 0)) -> Grid:
    """Grid description (ccfv_grid).  source=SRC_GAUSSIAN adds
    f = p0 exp(-((x-p1)^2 + (y-p2)^2) / p3) cos(p4 t), source_params = p."""
    ny = nx if ny is None else ny
    if domain is None:
        domain = (-1.0, 1.0, -1.0, 1.0) if bc == BC_COMPAT else (0.0, 1.0, 0.0, 1.0)
    g = Grid()
    g.nx, g.ny = int(nx), int(ny)
    g.x_min, g.x_max, g.y_min, g.y_max = (float(v) for v in domain)
    g.bc, g.velocity, g.scheme = int(bc), int(velocity), int(scheme)
    for i in range(4):
        g.vel_params[i] = float(vel_params[i]) if i < len(vel_params) else 0.0
    g.K = float(K)
    g.source = int(source)
    for i in range(5):
        g.source_params[i] = float(source_params[i]) if i < len(source_params) else 0.0
    return g


def _stream_ptr(stream):
    if stream is None:
        try:
            import torch
            return C.c_void_p(torch.cuda.current_stream().cuda_stream)
        except Exception:  # pragma: no cover - no torch / no GPU
            return C.c_void_p(0)
    if isinstance(stream, int):
        return C.c_void_p(stream)
    return C.c_void_p(stream.cuda_stream)


def _dptr(t):
    """Device pointer of a contiguous float64 CUDA tensor."""
    import torch
    if not (isinstance(t, torch.Tensor) and t.is_cuda and t.dtype == torch.float64
            and t.is_contiguous()):
        raise TypeError("expected a contiguous float64 CUDA tensor")
    return C.c_void_p(t.data_ptr())


class Solver:
    """A solver context (ccfv_create) for one grid on one device."""

    def __init__(self, grid: Grid, device: int = 0):
        self.grid = grid
        self.device = device
        h = C.c_void_p()
        rc = lib().ccfv_create(C.byref(h), C.byref(grid), device)
        if rc:
            raise CcfvError(rc, lib().ccfv_strerror(rc).decode())
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            lib().ccfv_destroy(self._h)
            self._h = None

    def __del__(self):  # pragma: no cover
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    def _chk(self, rc):
        if rc:
            msg = lib().ccfv_last_error(self._h).decode() or lib().ccfv_strerror(rc).decode()
            raise CcfvError(rc, msg)

    # -- time stepping -------------------------------------------------
    def step(self, C_dev, tn, dt, stream=None):
        self._chk(lib().ccfv_step(self._h, _dptr(C_dev), tn, dt, _stream_ptr(stream)))

    def fine(self, C_dev, tn, DT, J, stream=None):
        self._chk(lib().ccfv_fine(self._h, _dptr(C_dev), tn, DT, int(J), _stream_ptr(stream)))

    def coarse(self, C_dev, tn, DT, m=1, precision=FP64, stream=None, theta=0.5):
        """m coarse steps of DT/m; `theta` the implicit diffusion weight
        (0.5 Crank-Nicolson as the reference, COARSE_THETA_AUTO, or (0.5, 1])."""
        if theta == 0.5:
            self._chk(lib().ccfv_coarse(self._h, _dptr(C_dev), tn, DT, int(m), int(precision),
                                        _stream_ptr(stream)))
        else:
            self._chk(lib().ccfv_coarse_ex(self._h, _dptr(C_dev), tn, DT, int(m),
                                           int(precision), float(theta), _stream_ptr(stream)))

    def run(self, field, t0, dt, nsteps, stream=None):
        """Serial steps; `field` is a CUDA tensor (in place) or a numpy array
        (host memory, returns a new array)."""
        if isinstance(field, np.ndarray):
            c = np.ascontiguousarray(field, dtype=np.float64).copy()
            self._chk(lib().ccfv_run(self._h, C_void(c), MEM_HOST, t0, dt, int(nsteps),
                                     _stream_ptr(stream)))
            return c
        self._chk(lib().ccfv_run(self._h, _dptr(field), MEM_DEVICE, t0, dt, int(nsteps),
                                 _stream_ptr(stream)))
        return field

    def check(self, stream=None):
        self._chk(lib().ccfv_check(self._h, _stream_ptr(stream)))

    def fine_slices(self, fields, t0, slice_dt, DT, J, stream=None):
        """F on every field of a (n, nx, ny) CUDA tensor, in place."""
        self._chk(lib().ccfv_fine_slices(self._h, _dptr(fields), int(fields.shape[0]), t0,
                                         slice_dt, DT, int(J), _stream_ptr(stream)))

    def correct(self, form, U, F, W, Gold=None, stream=None):
        """Parareal correction of one slice; returns (sum dU^2, sum U^2)."""
        a, b = C.c_double(), C.c_double()
        self._chk(lib().ccfv_correct(self._h, int(form), _dptr(U), _dptr(F),
                                     None if Gold is None else _dptr(Gold), _dptr(W),
                                     C.byref(a), C.byref(b), _stream_ptr(stream)))
        return a.value, b.value

    def autotune(self, dt, precision=FP64, stream=None) -> int:
        seg = C.c_int(0)
        self._chk(lib().ccfv_autotune(self._h, dt, int(precision), C.byref(seg),
                                      _stream_ptr(stream)))
        return seg.value

    SWEEP_NAMES = ("general", "uniform", "filter", "source", "filter_exact", "cell",
                   "cell_exact", "cell_compat")

    def sweep_plan(self, dt, precision=FP64):
        """Kernel variant and segment length of the three sub-steps of a step
        of dt: [(variant name, cells per CTA)] * 3."""
        v, sg = (C.c_int * 3)(), (C.c_int * 3)()
        self._chk(lib().ccfv_sweep_plan(self._h, dt, int(precision), v, sg))
        return [(self.SWEEP_NAMES[v[i]], sg[i]) for i in range(3)]

    SWEEP_KERNELS = {"general": "sweep_kernel", "uniform": "sweep_fast_kernel",
                     "filter": "sweep_filter_kernel", "source": "sweep_kernel",
                     "filter_exact": "sweep_filter_kernel", "cell": "sweep_filter_kernel",
                     "cell_exact": "sweep_filter_kernel", "cell_compat": "sweep_filter_kernel"}

    def variant_names(self, dt, precision=FP64):
        """Names of the sweep kernels a step of dt launches (x, y, x)."""
        return "/".join(self.SWEEP_KERNELS[n] for n, _ in self.sweep_plan(dt, precision))

    # -- fields and diagnostics --------------------------------------------
    def exact_ref(self, C_dev, t, stream=None):
        self._chk(lib().ccfv_exact_ref(self._h, _dptr(C_dev), t, _stream_ptr(stream)))

    def gaussians(self, C_dev, params, images=0, stream=None):
        p = np.ascontiguousarray(params, dtype=np.float64).reshape(-1, 4)
        self._chk(lib().ccfv_gaussians(self._h, _dptr(C_dev), p.shape[0], C_void(p),
                                       int(images), _stream_ptr(stream)))

    def error_norms(self, a, b, stream=None):
        r, m = C.c_double(), C.c_double()
        self._chk(lib().ccfv_error_norms(self._h, _dptr(a), _dptr(b), C.byref(r), C.byref(m),
                                         _stream_ptr(stream)))
        return r.value, m.value

    # -- Parareal --------------------------------------------------------
    def parareal(self, C0, C_T=None, *, t0, t1, nt_fine, n_slices, coarse_ratio=0, tol=0.0,
                 kmax=8, coarse_precision=FP64, form=FORM_STANDARD, ref=None, coarse_theta=0.5,
                 stream=None):
        """Parareal solve.  C0 / C_T are CUDA tensors (device) or numpy
        arrays (host); `ref` an optional CUDA tensor the iterates at t1 are
        compared with; `coarse_theta` the implicit weight of the coarse
        propagator's diffusion (0.5 Crank-Nicolson as the reference, 1
        backward Euler).  Returns (C_T, stats dict)."""
        host = isinstance(C0, np.ndarray)
        o = PararealOpts(t0, t1, int(nt_fine), int(n_slices), int(coarse_ratio), float(tol),
                         int(kmax), int(coarse_precision), int(form),
                         MEM_HOST if host else MEM_DEVICE,
                         None if ref is None else _dptr(ref).value, float(coarse_theta))
        st = Stats()
        if host:
            c0 = np.ascontiguousarray(C0, dtype=np.float64)
            out = np.empty_like(c0) if C_T is None else C_T
            rc = lib().ccfv_parareal(self._h, C.byref(o), C_void(c0), C_void(out), C.byref(st),
                                     _stream_ptr(stream))
        else:
            import torch
            out = torch.empty_like(C0) if C_T is None else C_T
            rc = lib().ccfv_parareal(self._h, C.byref(o), _dptr(C0), _dptr(out), C.byref(st),
                                     _stream_ptr(stream))
        self._chk(rc)
        return out, st.as_dict()


def _problem(p):
    """ctypes Problem from a dict (grid, C0, C_T, Parareal options)."""
    host = isinstance(p["C0"], np.ndarray)
    o = PararealOpts(p["t0"], p["t1"], int(p["nt_fine"]), int(p["n_slices"]),
                     int(p.get("coarse_ratio", 0)), float(p.get("tol", 0.0)),
                     int(p.get("kmax", 8)), int(p.get("coarse_precision", FP64)),
                     int(p.get("form", FORM_STANDARD)), MEM_HOST if host else MEM_DEVICE, None,
                     float(p.get("coarse_theta", 0.5)))
    pr = Problem()
    pr.grid = p["grid"]
    pr.opts = o
    if host:
        pr.C0 = p["C0"].ctypes.data
        pr.C_T = p["C_T"].ctypes.data
    else:
        pr.C0 = _dptr(p["C0"]).value
        pr.C_T = _dptr(p["C_T"]).value
    return pr


class Server:
    """Continuous-batching request loop (ccfv_server_*).  Problems are dicts
    as for batch_solve; C0 / C_T (host numpy or device tensors) must stay
    alive until the request completes."""

    def __init__(self, hbm_budget_bytes, device=0, max_active=0):
        self._h = C.c_void_p()
        o = ServerOpts(int(device), int(hbm_budget_bytes), int(max_active))
        rc = lib().ccfv_server_create(C.byref(self._h), C.byref(o))
        if rc:
            raise CcfvError(rc, lib().ccfv_strerror(rc).decode())
        self._keep = {}

    def submit(self, problem) -> int:
        t = C.c_uint64()
        rc = lib().ccfv_server_submit(self._h, C.byref(_problem(problem)), C.byref(t))
        if rc:
            raise CcfvError(rc, lib().ccfv_strerror(rc).decode())
        self._keep[t.value] = problem
        return t.value

    def poll(self, ticket):
        st, s, lat = C.c_int(), Stats(), C.c_double()
        rc = lib().ccfv_server_poll(self._h, ticket, C.byref(st), C.byref(s), C.byref(lat))
        return rc, st.value, (s.as_dict() if st.value == REQ_DONE else None), lat.value

    def wait(self, ticket, timeout_s=0.0):
        s, lat = Stats(), C.c_double()
        rc = lib().ccfv_server_wait(self._h, ticket, float(timeout_s), C.byref(s), C.byref(lat))
        if rc:
            raise CcfvError(rc, lib().ccfv_strerror(rc).decode())
        self._keep.pop(ticket, None)
        return s.as_dict(), lat.value

    def cancel(self, ticket):
        return lib().ccfv_server_cancel(self._h, ticket)

    def info(self):
        u, a, q = C.c_size_t(), C.c_int(), C.c_int()
        lib().ccfv_server_info(self._h, C.byref(u), C.byref(a), C.byref(q))
        return dict(used_bytes=u.value, active=a.value, queued=q.value)

    def close(self):
        if self._h:
            lib().ccfv_server_destroy(self._h)
            self._h = None

    def __del__(self):  # pragma: no cover
        try:
            self.close()
        except Exception:
            pass


def coarse_theta(grid, *, t0, t1, nt_fine, n_slices, coarse_ratio=0, coarse_theta=0.5):
    """The coarse diffusion weight a Parareal run with these options uses on
    `grid` (COARSE_THETA_AUTO resolved); no device work."""
    o = PararealOpts(t0, t1, int(nt_fine), int(n_slices), int(coarse_ratio), 0.0, 1, FP64,
                     FORM_DELTA, MEM_DEVICE, None, float(coarse_theta))
    th = C.c_double()
    rc = lib().ccfv_coarse_theta(C.byref(grid), C.byref(o), C.byref(th))
    if rc:
        raise CcfvError(rc, lib().ccfv_strerror(rc).decode())
    return th.value


def batch_solve(problems, device=0, stream=None):
    """Solve several Parareal problems together (ccfv_batch_solve).

    `problems` is a list of dicts with keys grid (Grid), C0, C_T (CUDA
    tensors or numpy arrays, all problems alike) and the Parareal options of
    Solver.parareal.  Returns the list of stats dicts."""
    n = len(problems)
    arr = (Problem * n)()
    keep = []
    for i, p in enumerate(problems):
        host = isinstance(p["C0"], np.ndarray)
        o = PararealOpts(p["t0"], p["t1"], int(p["nt_fine"]), int(p["n_slices"]),
                         int(p.get("coarse_ratio", 0)), float(p.get("tol", 0.0)),
                         int(p.get("kmax", 8)), int(p.get("coarse_precision", FP64)),
                         int(p.get("form", FORM_STANDARD)), MEM_HOST if host else MEM_DEVICE,
                         None, float(p.get("coarse_theta", 0.5)))
        arr[i].grid = p["grid"]
        arr[i].opts = o
        if host:
            c0 = np.ascontiguousarray(p["C0"], dtype=np.float64)
            keep.append(c0)
            arr[i].C0 = c0.ctypes.data
            arr[i].C_T = p["C_T"].ctypes.data
        else:
            arr[i].C0 = _dptr(p["C0"]).value
            arr[i].C_T = _dptr(p["C_T"]).value
    st = (Stats * n)()
    rc = lib().ccfv_batch_solve(n, arr, st, int(device), _stream_ptr(stream))
    if rc:
        raise CcfvError(rc, lib().ccfv_strerror(rc).decode())
    return [st[i].as_dict() for i in range(n)]


def C_void(a: np.ndarray):
    return C.c_void_p(a.ctypes.data)


# ---------------------------------------------------------------------------
# Reference-shaped interface (T2S4_Parareal.cu:724-984).

class GPUContext:
    """State of one solve: grid parameters and the device field v_d_Cn
    (struct GPUContext, T2S4_Parareal.cu:724-768).  Scratch buffers are owned
    by the library context instead of 40 separate device arrays."""

    def __init__(self, Nx, Ny=None, K=0.0, *, bc=BC_COMPAT, velocity=VEL_REF_ROT4,
                 vel_params=(0, 0, 0, 0), domain=None, scheme=SCHEME_REFERENCE, device=0):
        import torch
        self.Nx = int(Nx)
        self.Ny = int(Nx if Ny is None else Ny)
        self.K = float(K)
        self.grid = make_grid(self.Nx, self.Ny, bc=bc, velocity=velocity, vel_params=vel_params,
                              K=K, domain=domain, scheme=scheme)
        self.dx = (self.grid.x_max - self.grid.x_min) / self.Nx
        self.dy = (self.grid.y_max - self.grid.y_min) / self.Ny
        self.N_grid = self.Nx * self.Ny
        self.solver = Solver(self.grid, device)
        self.v_d_Cn = torch.zeros(self.Nx, self.Ny, dtype=torch.float64,
                                  device=f"cuda:{device}")


def GpuOneStep(ctx: GPUContext, tn: float, dt: float) -> None:
    """One split step on ctx.v_d_Cn (GpuOneStep, T2S4_Parareal.cu:785-968)."""
    ctx.solver.step(ctx.v_d_Cn, tn, dt)


def CoarsePropagator(ctx: GPUContext, tn: float, DT: float) -> None:
    """One step of DT (CoarsePropagator, T2S4_Parareal.cu:971-974)."""
    ctx.solver.coarse(ctx.v_d_Cn, tn, DT, 1, FP64)


def FinePropagator(ctx: GPUContext, tn: float, DT: float, J: int) -> None:
    """J steps of DT/J (FinePropagator, T2S4_Parareal.cu:977-984)."""
    ctx.solver.fine(ctx.v_d_Cn, tn, DT, J)


def header_functions() -> list[str]:
    """Names of the functions declared in include/ccfv.h."""
    import re
    txt = HEADER.read_text()
    return sorted(set(re.findall(r"^\s*(?:const\s+)?[a-z_0-9]+\s+\**\s*(ccfv_[a-z_0-9]+)\s*\(",
                                 txt, re.M)))


__all__ = [n for n in dir() if not n.startswith("_")]
_ = os  # keep import for users that patch LIB_PATH via environment
