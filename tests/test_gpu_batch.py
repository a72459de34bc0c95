"""Batched solves (ccfv_batch_solve): each problem's result in the mix equals
the same problem solved alone through ccfv_parareal, within the FP64 parity
tolerance, for mixed sizes (tile tails, cluster sizes), velocities, forms
and coarse precisions."""
import numpy as np
import pytest

from conftest import periodic_field, rel_l2

pytestmark = pytest.mark.gpu
SRC = (2.0, 0.4, 0.6, 0.03, 5.0)


def dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).cuda()


def _problems(ccfv):
    rng = np.random.default_rng(42)
    specs = [
        # N, velocity, vel params, K, slices, nt, ratio, precision, form, tol
        (64, 1, (1.0, -0.5), 1e-2, 8, 64, 2, 0, 1, 0.0),
        (100, 1, (-0.7, 1.3), 1e-3, 10, 80, 4, 1, 1, 0.0),
        (256, 2, (2 * np.pi, 0.5, 0.5), 1e-3, 16, 256, 4, 0, 0, 0.0),
        (300, 1, (0.3, 0.4), 1e-4, 6, 60, 2, 0, 1, 0.0),
        (48, 3, (1.5,), 1e-3, 4, 32, 2, 0, 1, 0.0),
        (520, 2, (2 * np.pi, 0.5, 0.5), 5e-4, 8, 128, 4, 1, 1, 0.0),
        # with a Gaussian source: delta form (increments through G without
        # it) in FP64 and FP32, standard form
        (96, 2, (2 * np.pi, 0.5, 0.5), 1e-3, 8, 64, 2, 0, 1, 0.0, SRC),
        (80, 1, (0.8, -0.4), 1e-3, 8, 64, 2, 1, 1, 0.0, SRC),
        (72, 2, (2 * np.pi, 0.5, 0.5), 1e-3, 6, 48, 2, 0, 0, 0.0, SRC),
    ]
    probs = []
    for N, vel, vp, K, S, nt, ratio, prec, form, tol, *src in specs:
        g = ccfv.make_grid(N, bc=1, velocity=vel, vel_params=vp, K=K, scheme=1,
                           source=1 if src else 0,
                           source_params=src[0] if src else (0, 0, 0, 1, 0))
        C0 = periodic_field(N, int(rng.integers(1000)))
        probs.append(dict(grid=g, C0=C0, t0=0.0, t1=0.25, nt_fine=nt, n_slices=S,
                          coarse_ratio=ratio, tol=tol, kmax=3, coarse_precision=prec, form=form))
    # stiff diffusion (K dtc/h^2 of 5 - 13) with damped coarse steps: the
    # automatic weight in FP32 (delta form) and a fixed 0.8 in FP64 (standard)
    for N, K, prec, form, th in ((64, 5e-2, 1, 1, ccfv.COARSE_THETA_AUTO), (90, 2e-2, 0, 0, 0.8)):
        g = ccfv.make_grid(N, bc=1, velocity=1, vel_params=(0.6, -0.4), K=K, scheme=1)
        probs.append(dict(grid=g, C0=periodic_field(N, int(rng.integers(1000))), t0=0.0, t1=0.25,
                          nt_fine=64, n_slices=8, coarse_ratio=2, tol=0.0, kmax=3,
                          coarse_precision=prec, form=form, coarse_theta=th))
    return probs


def test_batch_matches_individual_solves(ccfv):
    import torch
    probs = _problems(ccfv)
    alone = []
    for p in probs:
        s = ccfv.Solver(p["grid"])
        out, st = s.parareal(dev(p["C0"]), t0=p["t0"], t1=p["t1"], nt_fine=p["nt_fine"],
                             n_slices=p["n_slices"], coarse_ratio=p["coarse_ratio"],
                             tol=p["tol"], kmax=p["kmax"], coarse_precision=p["coarse_precision"],
                             form=p["form"], coarse_theta=p.get("coarse_theta", 0.5))
        alone.append((out.cpu().numpy(), st))
    batch = []
    for p in probs:
        q = dict(p)
        q["C0"] = dev(p["C0"])
        q["C_T"] = torch.empty_like(q["C0"])
        batch.append(q)
    stats = ccfv.batch_solve(batch)
    torch.cuda.synchronize()
    for (ref, st_a), q, st_b in zip(alone, batch, stats):
        assert st_b["iterations"] == st_a["iterations"]
        assert rel_l2(q["C_T"].cpu().numpy(), ref) < 1e-12
        # the batched launches may split lines into other segment lengths
        # (tuned per line-length class): updates at the rounding level of the
        # converged solution differ in their last digits
        np.testing.assert_allclose(st_b["update"], st_a["update"], rtol=1e-6, atol=1e-11)


def test_batch_converges_per_instance(ccfv):
    """Instances stop independently when their own tolerance is met."""
    import torch
    probs = []
    for N, tol in ((128, 1e-10), (192, 1e-6)):
        g = ccfv.make_grid(N, bc=1, velocity=2, vel_params=(2 * np.pi, 0.5, 0.5), K=1e-3, scheme=1)
        C0 = periodic_field(N, 3)
        probs.append(dict(grid=g, C0=dev(C0), C_T=torch.empty(N, N, dtype=torch.float64,
                                                                device="cuda"),
                          t0=0.0, t1=0.5, nt_fine=4 * N // 2, n_slices=16, coarse_ratio=2,
                          tol=tol, kmax=16, coarse_precision=1, form=1))
    stats = ccfv.batch_solve(probs)
    for p, st in zip(probs, stats):
        assert st["converged"], st
        assert st["update"][-1] < p["tol"]
    assert stats[1]["iterations"] <= stats[0]["iterations"]


def test_resident_coarse_propagator_matches_shared_launches(ccfv, monkeypatch):
    """Small delta-form instances run their whole G phase in one CTA with the
    coarse field in shared memory (uniform and per-cell velocity fields, FP32
    and FP64 coarse steps, weak and stiff diffusion: the line's periodic
    system closed exactly); the results equal those of the shared coarse
    launches (CCFV_RESIDENT_G=0) within the FP64 parity tolerance."""
    import torch
    rng = np.random.default_rng(7)
    specs = [  # N, velocity, params, K, prec
        (64, 1, (1.0, -0.5), 1e-3, 1), (96, 2, (2 * np.pi, 0.5, 0.5), 1e-3, 0),
        (120, 3, (1.5,), 5e-4, 1), (80, 3, (1.5,), 2e-3, 0), (200, 1, (0.4, 0.9), 1e-4, 1),
        (72, 1, (0.6, -0.4), 5e-2, 1)]
    def probs():
        out = []
        for N, vel, vp, K, prec in specs:
            g = ccfv.make_grid(N, bc=1, velocity=vel, vel_params=vp, K=K, scheme=1)
            C0 = dev(periodic_field(N, int(rng.integers(1000))))
            out.append(dict(grid=g, C0=C0, C_T=torch.empty_like(C0), t0=0.0, t1=0.25,
                            nt_fine=64, n_slices=8, coarse_ratio=2, tol=0.0, kmax=4,
                            coarse_precision=prec, form=1,
                            coarse_theta=ccfv.COARSE_THETA_AUTO))
        return out
    a = probs()
    st_a = ccfv.batch_solve(a)
    monkeypatch.setenv("CCFV_RESIDENT_G", "0")
    b = [dict(p, C_T=torch.empty_like(p["C0"])) for p in a]
    st_b = ccfv.batch_solve(b)
    for p, q, x, y in zip(a, b, st_a, st_b):
        assert x["iterations"] == y["iterations"] == 4
        assert rel_l2(p["C_T"].cpu().numpy(), q["C_T"].cpu().numpy()) < 1e-12
        np.testing.assert_allclose(x["update"], y["update"], rtol=1e-5, atol=1e-11)
