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


def _simpson_cells(nx, dom, sp):
    """3x3 Simpson cell averages of f = a exp(-r^2/den) (no time factor)."""
    x0, x1, y0, y1 = dom
    dx, dy = (x1 - x0) / nx, (y1 - y0) / nx
    xc = x0 + (np.arange(nx) + 0.5) * dx
    yc = y0 + (np.arange(nx) + 0.5) * dy
    w = np.array([1.0, 4.0, 1.0]) / 6.0
    out = np.zeros((nx, nx))
    for a, ox in zip(w, (-0.5, 0.0, 0.5)):
        for b, oy in zip(w, (-0.5, 0.0, 0.5)):
            X = (xc + ox * dx)[:, None]
            Y = (yc + oy * dy)[None, :]
            out += a * b * sp[0] * np.exp(-((X - sp[1]) ** 2 + (Y - sp[2]) ** 2) / sp[3])
    return out


@pytest.mark.parametrize("scheme,factor", [(1, 1.0), (0, 2.0)], ids=["consistent", "reference"])
def test_source_without_transport(oracle, scheme, factor):
    """V = 0, K = 0: every sweep is the identity plus its source quadrature, so
    C(T) = C0 + T f_h for the consistent scheme.  The reference's RHS weighs
    the source 0.5 Dt in each of the three sub-steps (x_b_RHS_on_gpu,
    y_b_RHS_on_gpu, T2S4_Parareal.cu:564-613), which doubles it:
    C(T) = C0 + 2 T f_h."""
    N, T, n = 24, 0.3, 6
    sp = (1.5, 0.4, 0.6, 0.02, 0.0)
    g = oracle.grid(N, bc=1, vel=1, vp=(0.0, 0.0), K=0.0, scheme=scheme, src=1, sp=sp)
    C0 = periodic_field(N, 5)
    out = oracle.run(g, C0, 0.0, T / n, n)
    want = C0 + factor * T * _simpson_cells(N, (0.0, 1.0, 0.0, 1.0), sp)
    assert np.abs(out - want).max() < 1e-13


@pytest.mark.parametrize("bc", [0, 1])
def test_source_enters_linearly(oracle, bc):
    """The step is affine in (C, f): S(C0; f) = S(C0; 0) + S(0; f)."""
    N, dt = 20, 0.01
    sp = (2.0, 0.1 if bc == 0 else 0.55, 0.2 if bc == 0 else 0.45, 0.05, 3.0)
    kw = dict(K=2e-3, scheme=1)
    if bc == 1:
        kw.update(bc=1, vel=2, vp=(2 * np.pi, 0.5, 0.5))
    C0 = periodic_field(N, 8) if bc == 1 else seeded_field(N, 8)
    a = oracle.run(oracle.grid(N, src=1, sp=sp, **kw), C0, 0.1, dt, 3)
    b = oracle.run(oracle.grid(N, **kw), C0, 0.1, dt, 3)
    c = oracle.run(oracle.grid(N, src=1, sp=sp, **kw), np.zeros_like(C0), 0.1, dt, 3)
    assert np.abs(a - (b + c)).max() < 1e-12 * max(1.0, np.abs(a).max())


@pytest.mark.parametrize("form", [0, 1], ids=["standard", "delta"])
def test_parareal_with_source_converges_to_serial_fine(oracle, form):
    """With a source the coarse propagator is affine; the delta form moves
    increments with its linear part, so both forms reach the serial fine
    solve after as many iterations as slices."""
    N, T, nt, S = 20, 0.2, 40, 5
    sp = (3.0, 0.45, 0.55, 0.03, 6.0)
    g = oracle.grid(N, bc=1, vel=2, vp=(2 * np.pi, 0.5, 0.5), K=1e-3, scheme=1, src=1, sp=sp)
    C0 = periodic_field(N, 3)
    fine = oracle.run(g, C0, 0.0, T / nt, nt)
    UT, it, upd = oracle.parareal(g, C0, t0=0.0, t1=T, nt_fine=nt, n_slices=S,
                                  coarse_steps=2, tol=0.0, kmax=S, form=form)
    assert it == S
    assert rel_l2(UT, fine) < 1e-13


@pytest.mark.parametrize("theta", [0.5, 0.8, 1.0])
def test_theta_step_damps_grid_scale_mode_as_derived(oracle, theta):
    """Zero velocity: one split step multiplies the checkerboard mode by
    a(nu/2)^2 a(nu), a(nu) = (2/3 - 32/9 (1-theta) nu) / (2/3 + 4 theta nu),
    the amplification the automatic coarse weight is derived from."""
    N, K, dt = 32, 0.05, 0.02
    g = oracle.grid(N, bc=oracle.BC_PERIODIC, vel=oracle.VEL_CONST, vp=(0.0, 0.0), K=K,
                    threads=4, scheme=1, theta=theta)
    i = np.arange(N)
    C0 = np.where((i[:, None] + i[None, :]) % 2 == 0, 1.0, -1.0)
    out = oracle.step(g, C0, 0.0, dt)
    nu = K * dt * N * N

    def a(n):
        return (2 / 3 - 32 / 9 * (1 - theta) * n) / (2 / 3 + 4 * theta * n)

    np.testing.assert_allclose(out, a(nu / 2) ** 2 * a(nu) * C0, rtol=1e-10, atol=1e-14)


def test_auto_coarse_theta_restores_convergence(oracle):
    """Stiff diffusion (K dtc/h^2 = 6.4, one coarse step per slice, 64
    slices): Crank-Nicolson coarse steps stall Parareal; the automatic weight
    converges in a few iterations to the serial fine solve, its fixed point
    whatever G is."""
    N, S, K, V = 64, 64, 0.1, (1.0, 0.5)
    g = oracle.grid(N, bc=oracle.BC_PERIODIC, vel=oracle.VEL_CONST, vp=V, K=K, threads=8,
                    scheme=1)
    C0 = oracle.gaussians(g, [0.4, 0.7], [0.6, 0.3], [2 * 0.06 ** 2, 2 * 0.04 ** 2], [1.0, 0.5],
                          img=1)
    nt = 512  # dt = 1/512 (CFL 0.125), 8 fine steps per slice
    fine = oracle.run(g, C0, 0.0, 1.0 / nt, nt)
    kw = dict(t0=0.0, t1=1.0, nt_fine=nt, n_slices=S, coarse_steps=1, tol=1e-10, kmax=12,
              form=oracle.FORM_DELTA)
    _, it_cn, upd_cn = oracle.parareal(g, C0, **kw)
    assert upd_cn[-1] > 1e-6, upd_cn
    UT, it, upd = oracle.parareal(g, C0, coarse_theta=oracle.COARSE_THETA_AUTO, **kw)
    assert it <= 12 and upd[-1] < 1e-10, upd
    assert rel_l2(UT, fine) < 1e-9
