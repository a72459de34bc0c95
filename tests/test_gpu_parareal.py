"""Parareal engine through the C ABI against the oracle, the reference's
golden Parareal run and the serial fine solve."""
import json
import os
from pathlib import Path

import numpy as np
import pytest

from conftest import periodic_field, rel_l2

pytestmark = pytest.mark.gpu
THREADS = min(32, os.cpu_count() or 1)


def dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).cuda()


def test_reference_schedule_matches_golden(ccfv):
    """40 slices, 1 coarse step per slice, 3 fixed iterations, FP64 STANDARD:
    the reference's own Parareal run (T2S4_Parareal.cu:1249-1355)."""
    z = np.load(Path(__file__).parent / "golden" / "parareal_N24.npz")
    meta = json.loads(str(z["meta"]))
    s = ccfv.Solver(ccfv.make_grid(meta["N"], K=meta["K"]))
    UT, st = s.parareal(z["C0"], t0=meta["T_min"], t1=meta["T_max"], nt_fine=meta["Nt"],
                        n_slices=meta["n_slices"], kmax=meta["kmax"])
    assert st["iterations"] == meta["kmax"]
    assert rel_l2(UT, z["UT"]) < 1e-12
    assert abs(np.abs(UT - z["uref"]).max() - z["err"][-1]) < 1e-12 * np.abs(z["uref"]).max()


@pytest.mark.parametrize("form", [0, 1])
def test_parareal_matches_oracle(oracle, ccfv, form):
    N, T, nt, S, ratio = 40, 0.25, 96, 12, 4
    vp = (2 * np.pi, 0.5, 0.5)
    C0 = periodic_field(N, 6)
    g = oracle.grid(N, bc=1, vel=2, vp=vp, K=1e-3, threads=THREADS, scheme=1)
    ref, it_o, upd_o = oracle.parareal(g, C0, t0=0.0, t1=T, nt_fine=nt, n_slices=S,
                                       coarse_steps=(nt // S) // ratio, tol=0.0, kmax=4, form=form)
    s = ccfv.Solver(ccfv.make_grid(N, bc=1, velocity=2, vel_params=vp, K=1e-3, scheme=1))
    UT, st = s.parareal(dev(C0), t0=0.0, t1=T, nt_fine=nt, n_slices=S, coarse_ratio=ratio,
                        tol=0.0, kmax=4, form=form)
    assert rel_l2(UT.cpu().numpy(), ref) < 1e-12
    np.testing.assert_allclose(st["update"], upd_o, rtol=1e-6)


@pytest.mark.parametrize("prec", [0, 1])
def test_parareal_converges_to_serial_fine(oracle, ccfv, prec):
    """Converged Parareal (FP64 or FP32 coarse) equals the serial fine
    solve within its tolerance."""
    N, T, nt, S, ratio, tol = 128, 1.0, 512, 16, 4, 1e-10
    vp = (2 * np.pi, 0.5, 0.5)
    den = 2 * 0.05 ** 2  # Gaussian hump, sigma 0.05 at (0.5, 0.75), one revolution
    C0 = oracle.gaussians(oracle.grid(N, bc=1), [0.5], [0.75], [den], [1.0], img=1)
    s = ccfv.Solver(ccfv.make_grid(N, bc=1, velocity=2, vel_params=vp, K=1e-3, scheme=1))
    fine = s.run(C0, 0.0, T / nt, nt)
    UT, st = s.parareal(dev(C0), t0=0.0, t1=T, nt_fine=nt, n_slices=S, coarse_ratio=ratio,
                        tol=tol, kmax=S, coarse_precision=prec, form=ccfv.FORM_DELTA)
    assert st["converged"], st
    assert rel_l2(UT.cpu().numpy(), fine) < 10 * tol, st


@pytest.mark.parametrize("form", [0, 1])
def test_parareal_with_source_matches_oracle(oracle, ccfv, form):
    """Time-dependent Gaussian source; the delta form propagates increments
    with the source-free coarse step."""
    N, T, nt, S, ratio = 40, 0.25, 96, 12, 4
    vp, sp = (2 * np.pi, 0.5, 0.5), (2.0, 0.4, 0.6, 0.03, 5.0)
    C0 = periodic_field(N, 7)
    g = oracle.grid(N, bc=1, vel=2, vp=vp, K=1e-3, threads=THREADS, scheme=1, src=1, sp=sp)
    ref, it_o, upd_o = oracle.parareal(g, C0, t0=0.0, t1=T, nt_fine=nt, n_slices=S,
                                       coarse_steps=(nt // S) // ratio, tol=0.0, kmax=4, form=form)
    s = ccfv.Solver(ccfv.make_grid(N, bc=1, velocity=2, vel_params=vp, K=1e-3, scheme=1,
                                   source=1, source_params=sp))
    UT, st = s.parareal(dev(C0), t0=0.0, t1=T, nt_fine=nt, n_slices=S, coarse_ratio=ratio,
                        tol=0.0, kmax=4, form=form)
    assert rel_l2(UT.cpu().numpy(), ref) < 1e-12
    np.testing.assert_allclose(st["update"], upd_o, rtol=1e-6)


def test_parareal_with_source_fp32_coarse_converges(oracle, ccfv):
    """One revolution of a Gaussian hump under a pulsating Gaussian source:
    FP32-coarse delta-form Parareal converges to the serial fine solve."""
    N, T, nt, S, ratio, tol = 128, 1.0, 512, 16, 4, 1e-10
    vp, sp = (2 * np.pi, 0.5, 0.5), (1.0, 0.4, 0.6, 0.02, 2 * np.pi)
    s = ccfv.Solver(ccfv.make_grid(N, bc=1, velocity=2, vel_params=vp, K=1e-3, scheme=1,
                                   source=1, source_params=sp))
    C0 = oracle.gaussians(oracle.grid(N, bc=1), [0.5], [0.75], [2 * 0.05 ** 2], [1.0], img=1)
    fine = s.run(C0, 0.0, T / nt, nt)
    UT, st = s.parareal(dev(C0), t0=0.0, t1=T, nt_fine=nt, n_slices=S, coarse_ratio=ratio,
                        tol=tol, kmax=S, coarse_precision=1, form=1)
    assert st["converged"], st
    assert rel_l2(UT.cpu().numpy(), fine) < 10 * tol, st


def test_fp32_coarse_converges_like_fp64_for_advection(ccfv):
    """Constant velocity, weak diffusion, 64 slices: FP32 coarse Parareal
    needs no more than two iterations beyond the FP64 one (its first coarse
    sweep runs in FP64, so FP32 rounding never seeds the high-wavenumber
    modes that Parareal amplifies)."""
    N, S, ratio = 414, 64, 8
    V = (0.84, -0.16)
    dt = 0.8 / (N * 0.84)
    nt = int(np.ceil(1.0 / dt / (S * ratio))) * S * ratio
    s = ccfv.Solver(ccfv.make_grid(N, bc=1, velocity=1, vel_params=V, K=9e-4, scheme=1))
    import torch
    C0 = torch.empty(N, N, dtype=torch.float64, device="cuda")
    s.gaussians(C0, [[0.5, 0.5, 0.005, 1.0], [0.3, 0.7, 0.01, 0.6]], images=1)
    it = {}
    for prec in (0, 1):
        _, st = s.parareal(C0, t0=0.0, t1=1.0, nt_fine=nt, n_slices=S, coarse_ratio=ratio,
                           tol=1e-10, kmax=S, coarse_precision=prec, form=1)
        assert st["converged"], st
        it[prec] = st["iterations"]
    assert it[1] <= it[0] + 2, it


def _stiff_case(N, K, V, S, ratio):
    dt = 0.8 / (N * max(abs(V[0]), abs(V[1])))
    nt = int(np.ceil(1.0 / dt / (S * ratio))) * S * ratio
    return nt


@pytest.mark.parametrize("theta,form", [(0.8, 0), (-1.0, 1), (1.0, 1)],
                         ids=["fixed0.8-standard", "auto-delta", "euler-delta"])
def test_damped_coarse_matches_oracle(oracle, ccfv, theta, form):
    """Coarse steps with a theta-weighted diffusion (K dtc/h^2 = 6.4): the
    iterates and update norms equal the oracle's (same weight, same rule for
    the automatic one)."""
    N, S, ratio, K, V = 64, 16, 8, 0.1, (1.0, 0.5)
    nt = _stiff_case(N, K, V, S, ratio)
    C0 = periodic_field(N, 11)
    g = oracle.grid(N, bc=1, vel=1, vp=V, K=K, threads=THREADS, scheme=1)
    ref, it_o, upd_o = oracle.parareal(g, C0, t0=0.0, t1=1.0, nt_fine=nt, n_slices=S,
                                       coarse_steps=(nt // S) // ratio, tol=0.0, kmax=4,
                                       form=form, coarse_theta=theta)
    s = ccfv.Solver(ccfv.make_grid(N, bc=1, velocity=1, vel_params=V, K=K, scheme=1))
    UT, st = s.parareal(dev(C0), t0=0.0, t1=1.0, nt_fine=nt, n_slices=S, coarse_ratio=ratio,
                        tol=0.0, kmax=4, form=form, coarse_theta=theta)
    assert rel_l2(UT.cpu().numpy(), ref) < 1e-12
    np.testing.assert_allclose(st["update"], upd_o, rtol=1e-6)


@pytest.mark.parametrize("prec", [0, 1])
def test_auto_coarse_theta_converges_on_stiff_diffusion(ccfv, prec):
    """64 slices, one coarse step per slice, K dtc/h^2 = 6.4: with
    Crank-Nicolson coarse steps in FP32 Parareal stalls (FP32 rounding in the
    stiff modes grows from slice to slice); with the automatic weight it
    converges in a handful of iterations, in FP64 and in FP32, to the serial
    fine solve."""
    N, S, ratio, K, V, tol = 200, 64, 8, 0.01024, (1.99, 0.5), 1e-10
    nt = _stiff_case(N, K, V, S, ratio)
    s = ccfv.Solver(ccfv.make_grid(N, bc=1, velocity=1, vel_params=V, K=K, scheme=1))
    import torch
    C0 = torch.empty(N, N, dtype=torch.float64, device="cuda")
    s.gaussians(C0, [[0.4, 0.6, 2 * 0.05 ** 2, 1.0], [0.7, 0.3, 2 * 0.03 ** 2, 0.5]], images=1)
    fine = s.run(C0.cpu().numpy(), 0.0, 1.0 / nt, nt)
    _, st_cn = s.parareal(C0, t0=0.0, t1=1.0, nt_fine=nt, n_slices=S, coarse_ratio=ratio,
                          tol=tol, kmax=16, coarse_precision=prec, form=1)
    if prec == 1:
        assert not st_cn["converged"], st_cn["update"][:16]
    UT, st = s.parareal(C0, t0=0.0, t1=1.0, nt_fine=nt, n_slices=S, coarse_ratio=ratio,
                        tol=tol, kmax=16, coarse_precision=prec, form=1,
                        coarse_theta=ccfv.COARSE_THETA_AUTO)
    assert st["converged"] and st["iterations"] <= 14, st["update"][:16]
    assert rel_l2(UT.cpu().numpy(), fine) < 10 * tol
