"""ctypes binding of the CPU oracle (liboracle.so) and of the reference
harness (_ref/libt2s4ref.so).

TEST INFRASTRUCTURE: imported only by the tests, the smoke check and the
benchmark's CPU-baseline / reference legs.  It is the checker, never the
thing measured as the product.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "liboracle.so"
REF_PATH = HERE / "_ref" / "libt2s4ref.so"

BC_COMPAT, BC_PERIODIC = 0, 1
VEL_REF_ROT4, VEL_CONST, VEL_ROTATION, VEL_SWIRL = 0, 1, 2, 3
FORM_STANDARD, FORM_DELTA = 0, 1
COARSE_THETA_AUTO = -1.0
SCHEME_REFERENCE, SCHEME_CONSISTENT = 0, 1
SRC_NONE, SRC_GAUSSIAN = 0, 1


class OrGrid(C.Structure):
    _fields_ = [
        ("nx", C.c_int), ("ny", C.c_int),
        ("x_min", C.c_double), ("x_max", C.c_double),
        ("y_min", C.c_double), ("y_max", C.c_double),
        ("bc", C.c_int), ("vel", C.c_int),
        ("vp", C.c_double * 4),
        ("K", C.c_double),
        ("quirks", C.c_int), ("threads", C.c_int),
        ("scheme", C.c_int),
        ("src", C.c_int),
        ("sp", C.c_double * 5),
        ("theta", C.c_double),
    ]


class OrPararealOpts(C.Structure):
    _fields_ = [
        ("t0", C.c_double), ("t1", C.c_double),
        ("nt_fine", C.c_int), ("n_slices", C.c_int), ("coarse_steps", C.c_int),
        ("tol", C.c_double), ("kmax", C.c_int), ("form", C.c_int),
        ("coarse_theta", C.c_double),
    ]


_DP = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")


def build() -> None:
    """Compile liboracle.so with the Makefile beside this file."""
    subprocess.run(["make", "-s", "-C", str(HERE), "liboracle.so"], check=True)


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            build()
        L = C.CDLL(str(LIB_PATH))
        G = C.POINTER(OrGrid)
        L.or_step.argtypes = [G, _DP, C.c_double, C.c_double]
        L.or_run.argtypes = [G, _DP, C.c_double, C.c_double, C.c_int]
        L.or_fine.argtypes = [G, _DP, C.c_double, C.c_double, C.c_int]
        L.or_coarse.argtypes = [G, _DP, C.c_double, C.c_double, C.c_int]
        L.or_auto_theta.argtypes = [G, C.c_double]
        L.or_auto_theta.restype = C.c_double
        L.or_parareal_ref.argtypes = [G, _DP, C.c_double, C.c_double, C.c_int, C.c_int,
                                      C.c_int, C.c_void_p, C.c_void_p, _DP]
        L.or_parareal.argtypes = [G, C.POINTER(OrPararealOpts), _DP, _DP,
                                  C.POINTER(C.c_int), _DP]
        L.or_exact_ref.argtypes = [G, C.c_double, _DP]
        L.or_exact_ref.restype = None
        L.or_gaussians.argtypes = [G, C.c_int, _DP, _DP, _DP, _DP, C.c_int, _DP]
        L.or_gaussians.restype = None
        L.or_sum_kahan.argtypes = [_DP, C.c_long]
        L.or_sum_kahan.restype = C.c_double
        _lib = L
    return _lib


def grid(nx, ny=None, *, bc=BC_COMPAT, vel=VEL_REF_ROT4, vp=(0, 0, 0, 0), K=0.0,
         domain=None, quirks=1, threads=1, scheme=SCHEME_REFERENCE, src=SRC_NONE,
         sp=(0, 0, 0, 1, 0), theta=0.5) -> OrGrid:
    ny = nx if ny is None else ny
    if domain is None:
        domain = (-1.0, 1.0, -1.0, 1.0) if bc == BC_COMPAT else (0.0, 1.0, 0.0, 1.0)
    g = OrGrid()
    g.nx, g.ny = nx, ny
    g.x_min, g.x_max, g.y_min, g.y_max = domain
    g.bc, g.vel = bc, vel
    for i in range(4):
        g.vp[i] = float(vp[i]) if i < len(vp) else 0.0
    g.K = K
    g.quirks, g.threads = quirks, threads
    g.scheme = scheme
    g.src = src
    for i in range(5):
        g.sp[i] = float(sp[i]) if i < len(sp) else 0.0
    g.theta = float(theta)
    return g


def _chk(rc):
    if rc != 0:
        raise RuntimeError(f"oracle call failed with status {rc}")


def step(g, C0, tn, dt):
    c = np.array(C0, dtype=np.float64, order="C").reshape(-1).copy()
    _chk(lib().or_step(C.byref(g), c, tn, dt))
    return c.reshape(g.nx, g.ny)


def run(g, C0, t0, dt, nsteps):
    c = np.array(C0, dtype=np.float64, order="C").reshape(-1).copy()
    _chk(lib().or_run(C.byref(g), c, t0, dt, nsteps))
    return c.reshape(g.nx, g.ny)


def fine(g, C0, tn, DT, J):
    c = np.array(C0, dtype=np.float64, order="C").reshape(-1).copy()
    _chk(lib().or_fine(C.byref(g), c, tn, DT, J))
    return c.reshape(g.nx, g.ny)


def auto_theta(g, dtc):
    return lib().or_auto_theta(C.byref(g), dtc)


def coarse(g, C0, tn, DT, m=1, theta=None):
    """m coarse steps of DT/m; `theta` (None: the grid's own) the diffusion
    weight, COARSE_THETA_AUTO resolved for steps of DT/m."""
    if theta is not None:
        g = type(g).from_buffer_copy(g)
        g.theta = auto_theta(g, DT / max(m, 1)) if theta == COARSE_THETA_AUTO else theta
    c = np.array(C0, dtype=np.float64, order="C").reshape(-1).copy()
    _chk(lib().or_coarse(C.byref(g), c, tn, DT, m))
    return c.reshape(g.nx, g.ny)


def parareal_ref(g, C0, T_min, T_max, Nt, n_slices=40, kmax=8, Uref=None):
    c0 = np.ascontiguousarray(C0, dtype=np.float64).reshape(-1)
    UT = np.empty_like(c0)
    err = np.zeros(kmax)
    uref = None if Uref is None else np.ascontiguousarray(Uref, dtype=np.float64).reshape(-1)
    _chk(lib().or_parareal_ref(C.byref(g), c0, T_min, T_max, Nt, n_slices, kmax,
                               None if uref is None else uref.ctypes.data,
                               None if uref is None else err.ctypes.data, UT))
    return UT.reshape(g.nx, g.ny), err


def parareal(g, C0, *, t0, t1, nt_fine, n_slices, coarse_steps=1, tol=0.0, kmax=8,
             form=FORM_STANDARD, coarse_theta=0.5):
    o = OrPararealOpts(t0, t1, nt_fine, n_slices, coarse_steps, tol, kmax, form,
                       float(coarse_theta))
    c0 = np.ascontiguousarray(C0, dtype=np.float64).reshape(-1)
    UT = np.empty_like(c0)
    upd = np.zeros(max(kmax, 1))
    it = C.c_int(0)
    _chk(lib().or_parareal(C.byref(g), C.byref(o), c0, UT, C.byref(it), upd))
    return UT.reshape(g.nx, g.ny), it.value, upd[: it.value].copy()


def exact_ref(g, t):
    c = np.empty(g.nx * g.ny)
    lib().or_exact_ref(C.byref(g), t, c)
    return c.reshape(g.nx, g.ny)


def gaussians(g, cx, cy, den, amp, img=0):
    cx, cy, den, amp = (np.ascontiguousarray(a, dtype=np.float64) for a in (cx, cy, den, amp))
    c = np.empty(g.nx * g.ny)
    lib().or_gaussians(C.byref(g), len(cx), cx, cy, den, amp, img, c)
    return c.reshape(g.nx, g.ny)


def sum_kahan(a):
    a = np.ascontiguousarray(a, dtype=np.float64).reshape(-1)
    return lib().or_sum_kahan(a, a.size)


# ---------------------------------------------------------------------------
# The reference itself (GPU box only): _ref/libt2s4ref.so built by `make ref`.

_ref = None


def ref_available() -> bool:
    return REF_PATH.exists()


def ref():
    global _ref
    if _ref is None:
        L = C.CDLL(str(REF_PATH))
        L.ref_run.argtypes = [C.c_int, C.c_double, C.c_double, C.c_double, C.c_int, _DP, _DP]
        L.ref_time_run.argtypes = [C.c_int, C.c_double, C.c_double, C.c_double, C.c_int, _DP,
                                   _DP, C.POINTER(C.c_float)]
        L.ref_exact.argtypes = [C.c_int, C.c_double, C.c_double, _DP]
        L.ref_parareal.argtypes = [C.c_int, C.c_double, C.c_double, C.c_double, C.c_int, C.c_int,
                                   C.c_int, _DP, C.c_void_p, C.c_void_p, _DP]
        _ref = L
    return _ref


def ref_run(N, K, t0, dt, nsteps, C0):
    c0 = np.ascontiguousarray(C0, dtype=np.float64).reshape(-1)
    out = np.empty_like(c0)
    _chk(ref().ref_run(N, K, t0, dt, nsteps, c0, out))
    return out.reshape(N, N)


def ref_time_run(N, K, t0, dt, nsteps, C0):
    c0 = np.ascontiguousarray(C0, dtype=np.float64).reshape(-1)
    out = np.empty_like(c0)
    ms = C.c_float(0)
    _chk(ref().ref_time_run(N, K, t0, dt, nsteps, c0, out, C.byref(ms)))
    return out.reshape(N, N), ms.value


def ref_exact(N, K, t):
    out = np.empty(N * N)
    _chk(ref().ref_exact(N, K, t, out))
    return out.reshape(N, N)


def ref_parareal(N, K, T_min, T_max, Nt, C0, n_slices=40, kmax=8, Uref=None):
    c0 = np.ascontiguousarray(C0, dtype=np.float64).reshape(-1)
    UT = np.empty_like(c0)
    err = np.zeros(kmax)
    uref = None if Uref is None else np.ascontiguousarray(Uref, dtype=np.float64).reshape(-1)
    _chk(ref().ref_parareal(N, K, T_min, T_max, Nt, n_slices, kmax, c0,
                            None if uref is None else uref.ctypes.data,
                            None if uref is None else err.ctypes.data, UT))
    return UT.reshape(N, N), err


def cpu_count() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:  # pragma: no cover
        return os.cpu_count() or 1
