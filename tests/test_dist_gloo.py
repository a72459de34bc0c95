"""Slice-distributed Parareal (ccfv.dist) on CPU: two gloo ranks, the oracle
as the compute backend.  The pipelined exchange (boundary states, increments,
the max all-reduce of updates, the final broadcast) must reproduce the
single-process Parareal of the oracle."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

N, T, NT, S, RATIO, KMAX = 24, 0.25, 48, 6, 2, 4
VP = (2 * np.pi, 0.5, 0.5)
SP = (2.0, 0.4, 0.6, 0.04, 5.0)  # Gaussian source (time-dependent)


class OracleSlices:
    """Compute backend on the oracle (test only)."""

    def __init__(self, O, g, theta=0.5):
        self.O, self.g, self.theta = O, g, theta

    def zeros(self, n):
        return torch.zeros(n, self.g.nx, self.g.ny, dtype=torch.float64)

    def fine(self, fields, t0, slice_dt, DT, J):
        for i in range(fields.shape[0]):
            fields[i].copy_(torch.from_numpy(self.O.fine(self.g, fields[i].numpy(),
                                                         t0 + i * slice_dt, DT, J)))

    def coarse(self, field, t, DT, m):
        field.copy_(torch.from_numpy(self.O.coarse(self.g, field.numpy(), t, DT, m,
                                                   theta=self.theta)))

    def coarse_increment(self, field, t, DT, m):
        g = type(self.g).from_buffer_copy(self.g)
        g.src = 0
        field.copy_(torch.from_numpy(self.O.coarse(g, field.numpy(), t, DT, m,
                                                   theta=self.theta)))

    def correct(self, form, U, F, W, Gold=None):
        u, f, w = U.numpy(), F.numpy(), W.numpy()
        if form == 0:  # standard
            g = Gold.numpy()
            nv = w + (f - g)
            g[...] = w
        else:
            nv = f + w
        d = nv - u
        u[...] = nv
        if form != 0:
            w[...] = d
        return float((d * d).sum()), float((nv * nv).sum())


def _grid(O, src, K=1e-3):
    return O.grid(N, bc=1, vel=2, vp=VP, K=K, scheme=1, src=src, sp=SP)


def _worker(rank, world, port, form, src, q, K=1e-3, theta=0.5):
    import sys
    from pathlib import Path
    root = Path(__file__).resolve().parents[1]
    sys.path.insert(0, str(root / "oracle"))
    sys.path.insert(0, str(root / "parareal-cc-cfv-split-gpu_b200"))
    sys.path.insert(0, str(root / "tests"))
    import oracle as O
    from ccfv.dist import parareal_dist
    from conftest import periodic_field
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                            world_size=world)
    try:
        g = _grid(O, src, K)
        C0 = torch.from_numpy(periodic_field(N, 4))
        out, st = parareal_dist(OracleSlices(O, g, theta), C0, t0=0.0, t1=T, nt_fine=NT, n_slices=S,
                                coarse_ratio=RATIO, tol=0.0, kmax=KMAX, form=form)
        q.put((rank, out.numpy().copy(), st))
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("src", [0, 1], ids=["nosource", "source"])
@pytest.mark.parametrize("form", [1, 0], ids=["delta", "standard"])
def test_distributed_parareal_matches_single_process(oracle, form, src):
    from conftest import periodic_field
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, form, src, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=240) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    g = _grid(oracle, src)
    ref, it, upd = oracle.parareal(g, periodic_field(N, 4), t0=0.0, t1=T, nt_fine=NT,
                                   n_slices=S, coarse_steps=(NT // S) // RATIO, tol=0.0,
                                   kmax=KMAX, form=form)
    res.sort(key=lambda x: x[0])
    for rank, out, st in res:
        assert np.linalg.norm(out - ref) / np.linalg.norm(ref) < 1e-13
        assert st["iterations"] == KMAX
        np.testing.assert_allclose(st["update"], upd, rtol=1e-9)
    assert res[0][2]["slices"] == (0, 3) and res[1][2]["slices"] == (3, 6)


@pytest.mark.parametrize("theta", [0.8, -1.0], ids=["fixed0.8", "auto"])
def test_distributed_parareal_damped_coarse_matches_single_process(oracle, theta):
    """Damped coarse steps (stiff diffusion, K dtc/h^2 = 6: the automatic
    weight is ~0.79) through the slice-distributed driver: the backend's G
    carries the weight, the ranks reproduce the oracle's single-process run."""
    from conftest import periodic_field
    K = 0.5
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, 1, 0, q, K, theta)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=240) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    g = _grid(oracle, 0, K)
    m = (NT // S) // RATIO
    if theta == oracle.COARSE_THETA_AUTO:
        assert 0.7 < oracle.auto_theta(g, (T / S) / m) < 0.85
    ref, it, upd = oracle.parareal(g, periodic_field(N, 4), t0=0.0, t1=T, nt_fine=NT,
                                   n_slices=S, coarse_steps=m, tol=0.0, kmax=KMAX, form=1,
                                   coarse_theta=theta)
    for rank, out, st in sorted(res, key=lambda x: x[0]):
        assert np.linalg.norm(out - ref) / np.linalg.norm(ref) < 1e-13
        np.testing.assert_allclose(st["update"], upd, rtol=1e-9)
