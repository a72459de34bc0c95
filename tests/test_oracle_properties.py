"""Properties of the oracle's periodic / generic-velocity extension (no
reference counterpart): exact solutions, conservation, linearity, order,
Parareal convergence."""
import numpy as np
import pytest

from conftest import periodic_field, rel_l2, seeded_field


def _const_case(oracle, N, K, V=(1.0, 0.5), scheme=1):
    g = oracle.grid(N, bc=oracle.BC_PERIODIC, vel=oracle.VEL_CONST, vp=V, K=K, threads=4,
                    scheme=scheme)
    den = 2 * 0.1 ** 2
    C0 = oracle.gaussians(g, [0.5], [0.5], [den], [1.0], img=2)
    return g, C0, den


def test_periodic_const_matches_exact_gaussian(oracle):
    K, T, V = 0.01, 0.125, (1.0, 0.5)
    g, C0, den = _const_case(oracle, 64, K, V)
    dt = T / 256
    CT = oracle.run(g, C0, 0.0, dt, 256)
    ex = oracle.gaussians(g, [(0.5 + V[0] * T) % 1], [(0.5 + V[1] * T) % 1], [den + 4 * K * T],
                          [den / (den + 4 * K * T)], img=2)
    assert rel_l2(CT, ex) < 2e-4


def test_spatial_order_consistent_scheme(oracle):
    """4th order in space on a smooth constant-velocity case (small fixed dt)."""
    K, T, V = 0.01, 0.125, (1.0, 0.5)
    errs = []
    for N in (32, 64, 128):
        g, C0, den = _const_case(oracle, N, K, V)
        CT = oracle.run(g, C0, 0.0, T / 256, 256)
        ex = oracle.gaussians(g, [(0.5 + V[0] * T) % 1], [(0.5 + V[1] * T) % 1],
                              [den + 4 * K * T], [den / (den + 4 * K * T)], img=2)
        errs.append(rel_l2(CT, ex))
    orders = [np.log2(errs[i] / errs[i + 1]) for i in range(2)]
    assert min(orders) >= 3.9, (errs, orders)


@pytest.mark.parametrize("vel,vp", [(2, (2 * np.pi, 0.5, 0.5)), (3, (1.5,)), (1, (1.0, -0.7))])
def test_periodic_mass_conservation(oracle, vel, vp):
    g = oracle.grid(48, bc=oracle.BC_PERIODIC, vel=vel, vp=vp, K=1e-3, threads=4)
    C0 = periodic_field(48, 3)
    CT = oracle.run(g, C0, 0.0, 0.01, 20)
    m0, m1 = oracle.sum_kahan(C0), oracle.sum_kahan(CT)
    assert abs(m1 - m0) / abs(m0) < 1e-13


@pytest.mark.parametrize("bc", [0, 1])
def test_linearity(oracle, bc):
    g = oracle.grid(32, bc=bc, vel=0 if bc == 0 else 3, vp=(0, 0, 0, 0) if bc == 0 else (1.5,),
                    K=2e-3)
    a, b = seeded_field(32, 1), seeded_field(32, 2)
    if bc == 1:
        a, b = periodic_field(32, 1), periodic_field(32, 2)
    sa = oracle.step(g, a, 0.1, 0.01)
    sb = oracle.step(g, b, 0.1, 0.01)
    sab = oracle.step(g, 2.0 * a - 3.0 * b, 0.1, 0.01)
    assert rel_l2(sab, 2.0 * sa - 3.0 * sb) < 1e-13


def test_parareal_forms_converge_to_serial_fine(oracle):
    N, T, nt, S = 24, 0.2, 64, 8
    g = oracle.grid(N, bc=oracle.BC_PERIODIC, vel=oracle.VEL_ROTATION,
                    vp=(2 * np.pi, 0.5, 0.5), K=1e-3)
    C0 = periodic_field(N, 5)
    fine = oracle.run(g, C0, 0.0, T / nt, nt)
    for form in (oracle.FORM_STANDARD, oracle.FORM_DELTA):
        UT, iters, upd = oracle.parareal(g, C0, t0=0.0, t1=T, nt_fine=nt, n_slices=S,
                                         coarse_steps=2, tol=1e-12, kmax=S, form=form)
        assert rel_l2(UT, fine) < 1e-10, (form, iters, upd)
    # after S iterations Parareal is exact (finite termination)
    UT, iters, upd = oracle.parareal(g, C0, t0=0.0, t1=T, nt_fine=nt, n_slices=S,
                                     coarse_steps=1, tol=0.0, kmax=S, form=oracle.FORM_DELTA)
    assert rel_l2(UT, fine) < 1e-13
