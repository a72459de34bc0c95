"""Slice-distributed Parareal across ranks (one process per GPU).

Rank r owns a contiguous block of time slices.  Every iteration
  * the fine propagators of all owned slices advance together on the rank's
    GPU (ccfv_fine_slices): the F phases of all ranks run concurrently;
  * the coarse sweep is pipelined: rank r receives the corrected state of its
    first slice boundary from rank r-1, propagates and corrects its slices
    (ccfv_coarse + ccfv_correct) and sends its last boundary state on;
  * the ranks agree on convergence with one max all-reduce of the slice
    updates.
The only data exchanged is one N^2 state per rank boundary per iteration
(torch.distributed send/recv: NCCL over NVLink between GPUs, gloo on CPU).
The final state ends on the last rank and is broadcast to every rank.

The compute backend is pluggable (``CudaSlices`` runs libccfv); the
exchange and ordering logic is the same for any backend.  The delta form
propagates slice increments with the linear part of G: a backend whose grid
has a source term provides ``coarse_increment`` (G without the source).
The coarse diffusion weight (ccfv_parareal_opts::coarse_theta) is a property
of the backend's G (``CudaSlices(solver, coarse_theta=...)``).
"""
from __future__ import annotations

import math

import torch
import torch.distributed as dist

from . import FORM_DELTA, FORM_STANDARD, FP64, SRC_NONE, Solver


class CudaSlices:
    """Compute backend on libccfv for one grid on the rank's GPU."""

    def __init__(self, solver, coarse_theta=0.5, timed=False):
        self.s = solver
        self.nx, self.ny = solver.grid.nx, solver.grid.ny
        self.device = torch.device("cuda", solver.device)
        self._hom = None
        self.theta = coarse_theta
        # timed: CUDA events around every F phase (fine_phase_ms, fine_cells)
        self.timed = timed
        self._ev = []
        self.fine_cells = 0
        self.fine_sweeps = 0

    def zeros(self, n):
        return torch.zeros(n, self.nx, self.ny, dtype=torch.float64, device=self.device)

    def fine(self, fields, t0, slice_dt, DT, J):
        if self.timed:
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record()
        self.s.fine_slices(fields, t0, slice_dt, DT, J)
        if self.timed:
            b.record()
            self._ev.append((a, b))
            self.fine_cells += 3 * J * fields.shape[0] * self.nx * self.ny
            self.fine_sweeps += 3 * J

    def fine_phase_ms(self):
        """Device time of the F phases since the last reset (synchronises)."""
        torch.cuda.synchronize(self.device)
        return sum(a.elapsed_time(b) for a, b in self._ev)

    def reset_timers(self):
        self._ev = []
        self.fine_cells = 0
        self.fine_sweeps = 0

    def coarse(self, field, t, DT, m):
        self.s.coarse(field, t, DT, m, FP64, theta=self.theta)

    def coarse_increment(self, field, t, DT, m):
        if self.s.grid.source == SRC_NONE:
            return self.coarse(field, t, DT, m)
        if self._hom is None:
            g = type(self.s.grid).from_buffer_copy(self.s.grid)
            g.source = SRC_NONE
            self._hom = Solver(g, self.s.device)
        self._hom.coarse(field, t, DT, m, FP64, theta=self.theta)

    def correct(self, form, U, F, W, Gold=None):
        return self.s.correct(form, U, F, W, Gold)


def slice_block(n_slices: int, world: int, rank: int):
    """Contiguous block [lo, hi) of slices owned by `rank`."""
    base, extra = divmod(n_slices, world)
    lo = rank * base + min(rank, extra)
    return lo, lo + base + (1 if rank < extra else 0)


def parareal_dist(backend, C0, *, t0, t1, nt_fine, n_slices, coarse_ratio=0, tol=0.0, kmax=8,
                  form=FORM_DELTA, group=None):
    """Parareal over the ranks of `group`; returns (U(t1) on every rank, stats)."""
    R = dist.get_world_size(group)
    r = dist.get_rank(group)
    if n_slices < R or nt_fine % n_slices:
        raise ValueError("need n_slices >= ranks and nt_fine a multiple of n_slices")
    J = nt_fine // n_slices
    if coarse_ratio and J % coarse_ratio:
        raise ValueError("coarse_ratio must divide nt_fine / n_slices")
    m = J // coarse_ratio if coarse_ratio else 1
    DT = (t1 - t0) / n_slices
    lo, hi = slice_block(n_slices, R, r)
    n = hi - lo
    U = backend.zeros(n + 1)          # U[lo .. hi]
    Gold = backend.zeros(n + 1) if form == FORM_STANDARD else None
    W = backend.zeros(1)[0]

    def recv_left(dst):
        if r > 0:
            dist.recv(dst, src=r - 1, group=group)

    def send_right(src):
        if r < R - 1:
            dist.send(src.contiguous(), dst=r + 1, group=group)

    # k = 0: U[s+1] = G(U[s]) (T2S4_Parareal.cu:1271-1280), pipelined over ranks
    if r == 0:
        U[0].copy_(C0)
    recv_left(U[0])
    for i in range(n):
        W.copy_(U[i])
        backend.coarse(W, t0 + (lo + i) * DT, DT, m)
        U[i + 1].copy_(W)
        if Gold is not None:
            Gold[i + 1].copy_(W)
    send_right(U[n])

    updates, it, converged = [], 0, False
    F = backend.zeros(n)
    prev_first = U[0].clone()
    for k in range(1, kmax + 1):
        # F phase: all owned slices at once, concurrently on every rank
        F.copy_(U[:n])
        backend.fine(F, t0 + lo * DT, DT, DT, J)
        # G phase: new state of the first boundary from the left neighbour
        prev_first.copy_(U[0])
        recv_left(U[0])
        worst = 0.0
        if form == FORM_DELTA:
            g_inc = getattr(backend, "coarse_increment", backend.coarse)
            W.copy_(U[0] - prev_first)          # increment entering this block
            zero = (r == 0)                     # U[0] never changes: G(0) = 0
            for i in range(n):
                if zero:
                    W.zero_()
                    zero = False
                else:
                    g_inc(W, t0 + (lo + i) * DT, DT, m)
                du, uu = backend.correct(FORM_DELTA, U[i + 1], F[i], W)
                worst = max(worst, math.sqrt(du) / math.sqrt(uu) if uu > 0 else math.sqrt(du))
        else:
            for i in range(n):
                W.copy_(U[i])
                backend.coarse(W, t0 + (lo + i) * DT, DT, m)
                du, uu = backend.correct(FORM_STANDARD, U[i + 1], F[i], W, Gold[i + 1])
                worst = max(worst, math.sqrt(du) / math.sqrt(uu) if uu > 0 else math.sqrt(du))
        send_right(U[n])
        t = torch.tensor([worst], dtype=torch.float64, device=U.device)
        dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
        worst = float(t.item())
        updates.append(worst)
        it = k
        if tol > 0 and worst < tol:
            converged = True
            break
    out = U[n].clone()
    dist.broadcast(out, src=R - 1, group=group)
    return out, dict(iterations=it, converged=converged, update=updates, slices=(lo, hi))
