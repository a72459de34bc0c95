"""CUDA path (through the C ABI) against the reference's golden vectors and
the oracle.  Parity bar: 1e-12 relative L2 for FP64 (the oracle itself
agrees with the reference binary to ~1e-13)."""
import glob
import json
import os
from pathlib import Path

import numpy as np
import pytest

from conftest import periodic_field, rel_l2, seeded_field

pytestmark = pytest.mark.gpu
TOL = 1e-12
THREADS = min(32, os.cpu_count() or 1)
GOLDEN = sorted(glob.glob(str(Path(__file__).parent / "golden" / "*.npz")))


def _load(f):
    z = np.load(f)
    return json.loads(str(z["meta"])), z


def dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).cuda()


def host(t):
    return t.cpu().numpy()


@pytest.mark.parametrize("f", [g for g in GOLDEN if _load(g)[0]["kind"] in ("run", "ic_run")],
                         ids=lambda p: Path(p).stem)
def test_cuda_matches_reference_golden(ccfv, f):
    """GpuOneStep through the reference-shaped binding, on the reference's
    own outputs."""
    meta, z = _load(f)
    ctx = ccfv.GPUContext(meta["N"], K=meta["K"])
    ctx.v_d_Cn.copy_(dev(z["C0"]))
    for n in range(meta["nsteps"]):
        ccfv.GpuOneStep(ctx, meta["t0"] + n * meta["dt"], meta["dt"])
    ctx.solver.check()
    assert rel_l2(host(ctx.v_d_Cn), z["out"]) < TOL


def _compat_case(oracle, ccfv, nx, ny, K, dt, nsteps, seed, scheme=0):
    C0 = seeded_field(nx, seed, ny=ny)
    g = oracle.grid(nx, ny, K=K, threads=THREADS, scheme=scheme)
    ref = oracle.run(g, C0, 0.0, dt, nsteps)
    s = ccfv.Solver(ccfv.make_grid(nx, ny, K=K, scheme=scheme))
    c = dev(C0)
    s.run(c, 0.0, dt, nsteps)
    s.check()
    return host(c), ref


@pytest.mark.parametrize("nx,ny", [(4, 4), (5, 9), (37, 37), (100, 60), (256, 256), (257, 257),
                                   (300, 301), (600, 520), (1024, 1024)])
def test_compat_matches_oracle_sizes(oracle, ccfv, nx, ny):
    """Ragged sizes, tile tails (M % 16), cluster sizes 1..4."""
    dx = 2.0 / max(nx, ny)
    out, ref = _compat_case(oracle, ccfv, nx, ny, 1e-3, 0.1 * dx, 3, nx + ny)
    assert rel_l2(out, ref) < TOL


@pytest.mark.parametrize("N", [2048, 4096])
def test_compat_matches_oracle_cluster_8_16(oracle, ccfv, N):
    """Cluster sizes 8 and 16 (non-portable) for the longest lines."""
    out, ref = _compat_case(oracle, ccfv, N, N, 1e-4, 0.2 / N, 1, 11)
    assert rel_l2(out, ref) < TOL


@pytest.mark.parametrize("scheme", [0, 1])
@pytest.mark.parametrize("K,cfl", [(0.0, 0.5), (0.05, 0.5), (0.02, 3.3), (1.0, 1.0)])
def test_compat_diffusion_and_cfl(oracle, ccfv, scheme, K, cfl):
    """Both schemes, zero / strong diffusion, feet several cells away."""
    N = 64
    dt = cfl * (2.0 / N) / 4.0
    out, ref = _compat_case(oracle, ccfv, N, N, K, dt, 4, 7, scheme)
    assert rel_l2(out, ref) < TOL


PERIODIC = [
    ("const", 1, (1.0, -0.6)),
    ("rotation", 2, (2 * np.pi, 0.5, 0.5)),
    ("swirl", 3, (1.5,)),
    ("refrot", 0, ()),
]


@pytest.mark.parametrize("name,vel,vp", PERIODIC, ids=[p[0] for p in PERIODIC])
@pytest.mark.parametrize("nx,ny", [(64, 64), (96, 80), (512, 512)])
def test_periodic_matches_oracle(oracle, ccfv, name, vel, vp, nx, ny):
    K = 1e-3
    dt = 0.8 / max(nx, ny) / 3.2
    C0 = periodic_field(nx, 9, ny=ny)
    g = oracle.grid(nx, ny, bc=1, vel=vel, vp=vp, K=K, threads=THREADS, scheme=1)
    ref = oracle.run(g, C0, 0.3, dt, 3)
    s = ccfv.Solver(ccfv.make_grid(nx, ny, bc=1, velocity=vel, vel_params=vp, K=K, scheme=1))
    c = dev(C0)
    s.run(c, 0.3, dt, 3)
    s.check()
    assert rel_l2(host(c), ref) < TOL


def test_periodic_mass_conserved(oracle, ccfv):
    N = 256
    C0 = periodic_field(N, 4)
    s = ccfv.Solver(ccfv.make_grid(N, bc=1, velocity=2, vel_params=(2 * np.pi, 0.5, 0.5),
                                   K=1e-3, scheme=1))
    c = dev(C0)
    s.run(c, 0.0, 0.8 / N / np.pi, 64)
    m0, m1 = oracle.sum_kahan(C0), oracle.sum_kahan(host(c))
    assert abs(m1 - m0) / abs(m0) < 1e-13


def test_propagators_match_oracle(oracle, ccfv):
    N, K, tn, DT = 48, 2e-3, 0.05, 0.04
    C0 = seeded_field(N, 3)
    g = oracle.grid(N, K=K)
    ctx = ccfv.GPUContext(N, K=K)
    ctx.v_d_Cn.copy_(dev(C0))
    ccfv.FinePropagator(ctx, tn, DT, 5)
    assert rel_l2(host(ctx.v_d_Cn), oracle.fine(g, C0, tn, DT, 5)) < TOL
    ctx.v_d_Cn.copy_(dev(C0))
    ccfv.CoarsePropagator(ctx, tn, DT)
    assert rel_l2(host(ctx.v_d_Cn), oracle.coarse(g, C0, tn, DT, 1)) < TOL
    c = dev(C0)
    ctx.solver.coarse(c, tn, DT, 3)
    assert rel_l2(host(c), oracle.coarse(g, C0, tn, DT, 3)) < TOL


def test_fp32_coarse_close_to_fp64(ccfv):
    N = 128
    C0 = periodic_field(N, 2)
    s = ccfv.Solver(ccfv.make_grid(N, bc=1, velocity=3, vel_params=(1.5,), K=1e-3, scheme=1))
    a, b = dev(C0), dev(C0)
    s.coarse(a, 0.0, 0.05, 4, ccfv.FP64)
    s.coarse(b, 0.0, 0.05, 4, ccfv.FP32)
    assert rel_l2(host(b), host(a)) < 2e-6


def test_host_memory_run_matches_device(ccfv):
    N = 80
    C0 = seeded_field(N, 8)
    s = ccfv.Solver(ccfv.make_grid(N, K=1e-3))
    out_h = s.run(C0, 0.0, 0.002, 5)
    c = dev(C0)
    s.run(c, 0.0, 0.002, 5)
    assert np.array_equal(out_h, host(c))


@pytest.mark.parametrize("K", [1e-4, 1e-2, 0.5, 5.0])
@pytest.mark.parametrize("nx", [64, 300, 1024])
def test_periodic_solver_variants_match_oracle(oracle, ccfv, K, nx):
    """Weak diffusion takes the filter kernel (recurrences warmed up over
    J cells, |mu|^J below rounding), strong diffusion the exact chunked-scan
    kernel; both agree with the oracle's Sherman-Morrison cyclic solve."""
    vp = (0.9, -1.7)
    dt = 0.8 / nx / 1.7
    C0 = periodic_field(nx, 21)
    g = oracle.grid(nx, bc=1, vel=1, vp=vp, K=K, threads=THREADS, scheme=1)
    ref = oracle.run(g, C0, 0.0, dt, 2)
    s = ccfv.Solver(ccfv.make_grid(nx, bc=1, velocity=1, vel_params=vp, K=K, scheme=1))
    c = dev(C0)
    s.run(c, 0.0, dt, 2)
    s.check()
    assert rel_l2(host(c), ref) < TOL


@pytest.mark.parametrize("nx,K", [(2048, 1e-4), (2048, 1e-3), (4096, 1e-3)])
def test_periodic_filter_segments_match_oracle(oracle, ccfv, nx, K):
    """Filter kernel with 9 and 18 segments per line: single-field calls
    sweep out of place, so no segment reads what another one writes."""
    vp = (0.9, -1.7)
    dt = 0.8 / nx / 1.7
    C0 = periodic_field(nx, 22)
    g = oracle.grid(nx, bc=1, vel=1, vp=vp, K=K, threads=THREADS, scheme=1)
    ref = oracle.run(g, C0, 0.0, dt, 2)
    s = ccfv.Solver(ccfv.make_grid(nx, bc=1, velocity=1, vel_params=vp, K=K, scheme=1))
    assert all(v == "filter" for v, _ in s.sweep_plan(dt))
    c = dev(C0)
    s.run(c, 0.0, dt, 2)
    s.check()
    assert rel_l2(host(c), ref) < TOL


@pytest.mark.parametrize("nx,ny,K", [(96, 96, 0.3), (300, 200, 0.2), (1000, 520, 0.05),
                                     (2048, 64, 0.02), (544, 40, 0.05), (545, 40, 0.05)])
def test_periodic_exact_filter_matches_oracle(oracle, ccfv, nx, ny, K):
    """Strong diffusion (diffusion numbers 6 - 14: the recurrence warm-up
    would exceed 64 cells): the filter kernel's cluster form, 1 to 8
    segments per line, closes the periodic system exactly across them
    (whole 272-cell segments and a shorter last one, down to a single cell:
    544 = 2 x 272, 545 = 2 x 272 + 1)."""
    vp = (0.9, -1.7)
    dt = 0.8 / max(nx, ny) / 1.7
    C0 = periodic_field(nx, 23, ny=ny)
    g = oracle.grid(nx, ny, bc=1, vel=1, vp=vp, K=K, threads=THREADS, scheme=1)
    ref = oracle.run(g, C0, 0.0, dt, 2)
    s = ccfv.Solver(ccfv.make_grid(nx, ny, bc=1, velocity=1, vel_params=vp, K=K, scheme=1))
    assert "filter_exact" in [v for v, _ in s.sweep_plan(dt)]
    c = dev(C0)
    s.run(c, 0.0, dt, 2)
    s.check()
    out = host(c)
    assert rel_l2(out, ref) < TOL
    assert abs(out.sum() - C0.sum()) < 1e-12 * np.abs(C0).sum()


@pytest.mark.parametrize("nx,ny,K,form", [(64, 64, 1e-3, "cell"), (300, 260, 1e-4, "cell"),
                                          (2048, 40, 1e-3, "cell"), (4096, 24, 1e-4, "cell"),
                                          (96, 96, 0.3, "cell_exact"),
                                          (545, 40, 0.05, "cell_exact"),
                                          (1000, 520, 0.05, "cell_exact"),
                                          (2048, 64, 0.02, "cell_exact")])
def test_periodic_cell_filter_matches_oracle(oracle, ccfv, nx, ny, K, form):
    """Swirling deformation (feet differ from edge to edge): the filter
    kernel with the per-cell right-hand side, warm-up form (1 to 18 segments
    per line) and cluster form (strong diffusion), against the oracle's
    per-cell remap and Sherman-Morrison cyclic solve."""
    dt = 0.8 / max(nx, ny)
    C0 = periodic_field(nx, 31, ny=ny)
    g = oracle.grid(nx, ny, bc=1, vel=3, vp=(1.5,), K=K, threads=THREADS, scheme=1)
    ref = oracle.run(g, C0, 0.35, dt, 2)
    s = ccfv.Solver(ccfv.make_grid(nx, ny, bc=1, velocity=3, vel_params=(1.5,), K=K, scheme=1))
    assert form in [v for v, _ in s.sweep_plan(dt)]
    c = dev(C0)
    s.run(c, 0.35, dt, 2)
    s.check()
    out = host(c)
    assert rel_l2(out, ref) < TOL
    assert abs(out.sum() - C0.sum()) < 1e-12 * np.abs(C0).sum()


def test_fp32_cell_filter_coarse_close_to_fp64(ccfv):
    N = 256
    C0 = periodic_field(N, 14)
    s = ccfv.Solver(ccfv.make_grid(N, bc=1, velocity=3, vel_params=(1.5,), K=1e-3, scheme=1))
    assert "cell" in [v for v, _ in s.sweep_plan(0.01, ccfv.FP32)]
    a, b = dev(C0), dev(C0)
    s.coarse(a, 0.2, 0.02, 2, ccfv.FP64)
    s.coarse(b, 0.2, 0.02, 2, ccfv.FP32)
    assert rel_l2(host(b), host(a)) < 2e-6


def test_fp32_exact_filter_coarse_close_to_fp64(ccfv):
    N, K = 640, 0.05  # coarse steps of diffusion number ~60: the exact cluster form
    C0 = periodic_field(N, 13)
    s = ccfv.Solver(ccfv.make_grid(N, bc=1, velocity=1, vel_params=(0.6, 0.3), K=K, scheme=1))
    assert "filter_exact" in [v for v, _ in s.sweep_plan(0.003, ccfv.FP32)]
    a, b = dev(C0), dev(C0)
    s.coarse(a, 0.0, 0.006, 2, ccfv.FP64)
    s.coarse(b, 0.0, 0.006, 2, ccfv.FP32)
    # FP32 rounding (6e-8) grows with the condition number of the y sub-step's
    # cyclic system, (b + 2|a|) / (b - 2|a|) with a = 1/12 - nu/2, b = 10/12 + nu
    nu = K * 0.003 * N * N
    kappa = (10 / 12 + nu + 2 * abs(1 / 12 - nu / 2)) / (10 / 12 + nu - 2 * abs(1 / 12 - nu / 2))
    assert kappa > 100
    assert rel_l2(host(b), host(a)) < 6e-8 * kappa


def test_fp32_filter_coarse_close_to_fp64(ccfv):
    N = 256
    C0 = periodic_field(N, 12)
    s = ccfv.Solver(ccfv.make_grid(N, bc=1, velocity=2, vel_params=(2 * np.pi, 0.5, 0.5),
                                   K=1e-3, scheme=1))
    a, b = dev(C0), dev(C0)
    s.coarse(a, 0.0, 0.02, 2, ccfv.FP64)
    s.coarse(b, 0.0, 0.02, 2, ccfv.FP32)
    assert rel_l2(host(b), host(a)) < 2e-6


SRC_COMPAT = (1.5, 0.3, -0.2, 0.05, 4.0)   # on [-1, 1]^2
SRC_PERIODIC = (2.0, 0.4, 0.6, 0.03, 5.0)  # on [0, 1]^2


@pytest.mark.parametrize("scheme", [0, 1])
@pytest.mark.parametrize("N", [48, 300])
def test_compat_source_matches_oracle(oracle, ccfv, scheme, N):
    """Gaussian source: Simpson cell averages, f(t_a) remapped plus f(t_b) in
    the right-hand side of every sub-step, with either scheme's weight."""
    dt = 0.1 * (2.0 / N)
    C0 = seeded_field(N, 17)
    g = oracle.grid(N, K=1e-3, threads=THREADS, scheme=scheme, src=1, sp=SRC_COMPAT)
    ref = oracle.run(g, C0, 0.2, dt, 3)
    s = ccfv.Solver(ccfv.make_grid(N, K=1e-3, scheme=scheme, source=1, source_params=SRC_COMPAT))
    c = dev(C0)
    s.run(c, 0.2, dt, 3)
    s.check()
    assert rel_l2(host(c), ref) < TOL


@pytest.mark.parametrize("name,vel,vp", PERIODIC, ids=[p[0] for p in PERIODIC])
@pytest.mark.parametrize("scheme", [0, 1])
def test_periodic_source_matches_oracle(oracle, ccfv, name, vel, vp, scheme):
    nx, ny = 96, 80
    dt = 0.8 / nx / 3.2
    C0 = periodic_field(nx, 19, ny=ny)
    g = oracle.grid(nx, ny, bc=1, vel=vel, vp=vp, K=1e-3, threads=THREADS, scheme=scheme, src=1,
                    sp=SRC_PERIODIC)
    ref = oracle.run(g, C0, 0.1, dt, 3)
    s = ccfv.Solver(ccfv.make_grid(nx, ny, bc=1, velocity=vel, vel_params=vp, K=1e-3,
                                   scheme=scheme, source=1, source_params=SRC_PERIODIC))
    c = dev(C0)
    s.run(c, 0.1, dt, 3)
    s.check()
    assert rel_l2(host(c), ref) < TOL


def test_source_sweep_plan(ccfv):
    """A grid with a source runs the per-cell source kernel in every sub-step."""
    s = ccfv.Solver(ccfv.make_grid(128, bc=1, velocity=1, vel_params=(1.0, 0.5), K=1e-3,
                                   scheme=1, source=1, source_params=SRC_PERIODIC))
    assert [v for v, _ in s.sweep_plan(1e-3)] == ["source"] * 3
    s0 = ccfv.Solver(ccfv.make_grid(128, bc=1, velocity=1, vel_params=(1.0, 0.5), K=1e-3,
                                    scheme=1))
    assert [v for v, _ in s0.sweep_plan(1e-3)] == ["filter"] * 3


@pytest.mark.parametrize("theta,prec", [(0.8, 0), (-1.0, 0), (-1.0, 1)])
def test_coarse_ex_matches_oracle(oracle, ccfv, theta, prec):
    """ccfv_coarse_ex: coarse steps with a fixed or automatic diffusion weight
    (stiff: K dtc/h^2 = 12, automatic weight ~0.8) equal the oracle's."""
    N, K, DT, m = 120, 0.1, 0.02, 2
    vp = (0.7, -0.3)
    C0 = periodic_field(N, 31)
    g = oracle.grid(N, bc=1, vel=1, vp=vp, K=K, threads=THREADS, scheme=1)
    ref = oracle.coarse(g, C0, 0.1, DT, m, theta=theta)
    s = ccfv.Solver(ccfv.make_grid(N, bc=1, velocity=1, vel_params=vp, K=K, scheme=1))
    c = dev(C0)
    s.coarse(c, 0.1, DT, m, prec, theta=theta)
    s.check()
    assert rel_l2(host(c), ref) < (TOL if prec == 0 else 1e-5)
