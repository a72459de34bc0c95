"""CUDA path on the benchmark configurations and on the slice-distributed
building blocks.

* The small plain case: periodic 128^2, constant velocity (1, 1), nu = 0.01,
  Gaussian sigma = 0.1 at the centre, T = 1, fine dt at CFL 0.8 (160 steps),
  16 slices, one coarse step of 10 fine steps per slice, Parareal to 1e-10:
  the converged result against the serial fine solve, the oracle's Parareal
  and the exact shifted, diffused Gaussian.
* Spatial order of the CUDA path on a smooth constant-velocity case.
* The swirling-deformation velocity (per-cell feet) against the oracle on a
  2048^2 field for 8 steps.
* ccfv_fine_slices (in place, segments of a line in one thread-block
  cluster), ccfv_correct and the slice-distributed driver with one rank
  against ccfv_fine / ccfv_parareal.
"""
import os
import socket

import numpy as np
import pytest

from conftest import periodic_field, rel_l2

pytestmark = pytest.mark.gpu
THREADS = min(32, os.cpu_count() or 1)


def dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).cuda()


def host(t):
    return t.cpu().numpy()


def _small_plain_case(oracle, ccfv):
    N, K, T, V, sigma = 128, 0.01, 1.0, (1.0, 1.0), 0.1
    den = 2 * sigma ** 2
    g = ccfv.make_grid(N, bc=ccfv.BC_PERIODIC, velocity=ccfv.VEL_CONST, vel_params=V, K=K,
                       scheme=ccfv.SCHEME_CONSISTENT)
    s = ccfv.Solver(g)
    C0 = dev(np.zeros((N, N)))
    s.gaussians(C0, [[0.5, 0.5, den, 1.0]], images=2)
    # exact solution: the Gaussian moved by V T (one period: back to the centre)
    # and diffused, den -> den + 4 K T
    ex = dev(np.zeros((N, N)))
    s.gaussians(ex, [[(0.5 + V[0] * T) % 1.0, (0.5 + V[1] * T) % 1.0, den + 4 * K * T,
                      den / (den + 4 * K * T)]], images=2)
    nt = int(round(T / (0.8 * (1.0 / N) / max(V))))  # CFL 0.8: 160 steps
    return N, K, T, V, s, C0, ex, nt


def test_small_plain_parareal_converges_to_fine_and_exact(oracle, ccfv):
    N, K, T, V, s, C0, ex, nt = _small_plain_case(oracle, ccfv)
    assert nt == 160
    fine = C0.clone()
    s.run(fine, 0.0, T / nt, nt)
    out, st = s.parareal(C0, t0=0.0, t1=T, nt_fine=nt, n_slices=16, coarse_ratio=10, tol=1e-10,
                         kmax=16, coarse_precision=ccfv.FP64, form=ccfv.FORM_DELTA)
    s.check()
    assert st["converged"], st["update"]
    err_fine = rel_l2(host(out), host(fine))
    err_exact = rel_l2(host(out), host(ex))
    assert err_fine <= 1e-10, (err_fine, st["update"])
    # the scheme's own error at 128^2, CFL 0.8 (the oracle's serial fine run: 9.0e-6)
    assert err_exact < 2e-5, err_exact
    # against the oracle's Parareal on the same field (same schedule)
    g = oracle.grid(N, bc=1, vel=1, vp=V, K=K, threads=THREADS, scheme=1)
    ref, its, _ = oracle.parareal(g, host(C0), t0=0.0, t1=T, nt_fine=nt, n_slices=16,
                                  coarse_steps=1, tol=1e-10, kmax=16, form=oracle.FORM_DELTA)
    assert its == st["iterations"]
    assert rel_l2(host(out), ref) < 1e-12
    # FP32 coarse steps converge to the same fine solution
    out32, st32 = s.parareal(C0, t0=0.0, t1=T, nt_fine=nt, n_slices=16, coarse_ratio=10,
                             tol=1e-10, kmax=16, coarse_precision=ccfv.FP32,
                             form=ccfv.FORM_DELTA)
    assert st32["converged"]
    assert rel_l2(host(out32), host(fine)) <= 1e-10


def test_cuda_spatial_order_constant_velocity(ccfv):
    """Fourth order in space on a smooth constant-velocity case (fixed small
    dt so that the time error stays below the spatial error)."""
    K, T, V, sigma = 0.01, 0.125, (1.0, 0.5), 0.1
    den = 2 * sigma ** 2
    errs = []
    for N in (32, 64, 128):
        s = ccfv.Solver(ccfv.make_grid(N, bc=ccfv.BC_PERIODIC, velocity=ccfv.VEL_CONST,
                                       vel_params=V, K=K, scheme=ccfv.SCHEME_CONSISTENT))
        c = dev(np.zeros((N, N)))
        s.gaussians(c, [[0.5, 0.5, den, 1.0]], images=2)
        ex = dev(np.zeros((N, N)))
        s.gaussians(ex, [[(0.5 + V[0] * T) % 1, (0.5 + V[1] * T) % 1, den + 4 * K * T,
                          den / (den + 4 * K * T)]], images=2)
        s.run(c, 0.0, T / 256, 256)
        s.check()
        errs.append(rel_l2(host(c), host(ex)))
    orders = [np.log2(errs[i] / errs[i + 1]) for i in range(len(errs) - 1)]
    assert min(orders) >= 3.9, (errs, orders)


def test_swirl_matches_oracle_2048(oracle, ccfv):
    """Per-cell feet of the time-dependent swirling deformation on a 2048^2
    field, 8 steps at CFL 0.8, against the oracle."""
    N, K, nsteps = 2048, 1e-4, 8
    dt = 0.8 / N
    C0 = periodic_field(N, 12)
    g = oracle.grid(N, bc=1, vel=3, vp=(1.5,), K=K, threads=THREADS, scheme=1)
    ref = oracle.run(g, C0, 0.3, dt, nsteps)
    s = ccfv.Solver(ccfv.make_grid(N, bc=ccfv.BC_PERIODIC, velocity=ccfv.VEL_SWIRL,
                                   vel_params=(1.5,), K=K, scheme=ccfv.SCHEME_CONSISTENT))
    c = dev(C0)
    s.run(c, 0.3, dt, nsteps)
    s.check()
    assert rel_l2(host(c), ref) < 1e-12
    m0, m1 = oracle.sum_kahan(C0), oracle.sum_kahan(host(c))
    assert abs(m1 - m0) / abs(m0) < 1e-13


@pytest.mark.parametrize("nx,ny", [(4096, 32), (2048, 48), (300, 40)])
def test_fine_slices_match_fine_per_slice(ccfv, nx, ny):
    """ccfv_fine_slices sweeps its fields in place: the segments of a long
    line form one thread-block cluster whose CTAs all finish reading before
    any stores.  Each field must equal ccfv_fine on that field alone."""
    import torch
    g = ccfv.make_grid(nx, ny, bc=ccfv.BC_PERIODIC, velocity=ccfv.VEL_ROTATION,
                       vel_params=(2 * np.pi, 0.5, 0.5), K=1e-3,
                       scheme=ccfv.SCHEME_CONSISTENT)
    s = ccfv.Solver(g)
    n, J, t0 = 3, 2, 0.05
    dt = 0.8 / max(nx, ny) / np.pi
    DT = J * dt
    fields = torch.stack([dev(periodic_field(nx, 20 + i, ny=ny)) for i in range(n)])
    ref = [fields[i].clone() for i in range(n)]
    s.fine_slices(fields, t0, DT, DT, J)
    for i in range(n):
        s.fine(ref[i], t0 + i * DT, DT, J)
    s.check()
    for i in range(n):
        assert rel_l2(host(fields[i]), host(ref[i])) < 1e-12, i


@pytest.mark.parametrize("form", [0, 1], ids=["standard", "delta"])
def test_correct_matches_formula(ccfv, form):
    import torch
    N = 96
    s = ccfv.Solver(ccfv.make_grid(N, bc=ccfv.BC_PERIODIC, velocity=ccfv.VEL_CONST,
                                   vel_params=(1.0, 0.5), K=1e-3,
                                   scheme=ccfv.SCHEME_CONSISTENT))
    rng = np.random.default_rng(3)
    U0, F, W, G = (rng.standard_normal((N, N)) for _ in range(4))
    U, Fd, Wd = dev(U0), dev(F), dev(W)
    Gd = dev(G) if form == 0 else None
    du, uu = s.correct(form, U, Fd, Wd, Gd)
    new = W + (F - G) if form == 0 else F + W
    assert np.allclose(host(U), new, rtol=0, atol=1e-14)
    if form == 0:
        assert np.array_equal(host(Gd), W)
    else:
        assert np.allclose(host(Wd), new - U0, rtol=0, atol=1e-14)
    assert abs(du - float(((new - U0) ** 2).sum())) < 1e-9 * max(1.0, du)
    assert abs(uu - float((new ** 2).sum())) < 1e-9 * uu


def _free_port():
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        return sk.getsockname()[1]


@pytest.mark.parametrize("form", [1, 0], ids=["delta", "standard"])
def test_slice_distributed_one_rank_matches_parareal(ccfv, form):
    """ccfv.dist.parareal_dist with one rank (gloo, CUDA tensors) on the
    CudaSlices backend equals the single-process engine ccfv_parareal."""
    import torch.distributed as dist
    from ccfv.dist import CudaSlices, parareal_dist
    N, T, nt, S, ratio = 64, 0.25, 64, 8, 4
    g = ccfv.make_grid(N, bc=ccfv.BC_PERIODIC, velocity=ccfv.VEL_ROTATION,
                       vel_params=(2 * np.pi, 0.5, 0.5), K=1e-3,
                       scheme=ccfv.SCHEME_CONSISTENT)
    s = ccfv.Solver(g)
    C0 = dev(periodic_field(N, 7))
    ref, st = s.parareal(C0, t0=0.0, t1=T, nt_fine=nt, n_slices=S, coarse_ratio=ratio, tol=0.0,
                         kmax=4, coarse_precision=ccfv.FP64, form=form)
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{_free_port()}", rank=0,
                            world_size=1)
    try:
        out, dst = parareal_dist(CudaSlices(s), C0, t0=0.0, t1=T, nt_fine=nt, n_slices=S,
                                 coarse_ratio=ratio, tol=0.0, kmax=4, form=form)
    finally:
        dist.destroy_process_group()
    s.check()
    assert dst["iterations"] == st["iterations"] == 4
    assert rel_l2(host(out), host(ref)) < 1e-12
    np.testing.assert_allclose(dst["update"], st["update"], rtol=1e-6)
