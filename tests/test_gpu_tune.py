"""The line-tile autotuner (ccfv_autotune): the segment length it picks keeps
the oracle's result and is not slower than the default on a 1024^2 field."""
import os

import numpy as np
import pytest

from conftest import periodic_field, rel_l2

pytestmark = pytest.mark.gpu
THREADS = min(32, os.cpu_count() or 1)


def _time_steps(s, c, dt, n=24, reps=3):
    import torch
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s.run(c, 0.0, dt, 2)
    best = 1e30
    for _ in range(reps):
        a.record()
        s.run(c, 0.0, dt, n)
        b.record()
        torch.cuda.synchronize()
        best = min(best, a.elapsed_time(b))
    return best


def test_autotuned_segments_keep_parity_and_speed(oracle, ccfv):
    import torch
    N, K = 1024, 1e-3
    dt = 1.0 / (4 * N)
    g = ccfv.make_grid(N, bc=1, velocity=2, vel_params=(2 * np.pi, 0.5, 0.5), K=K, scheme=1)
    C0 = periodic_field(N, 17)
    s = ccfv.Solver(g)
    before = s.sweep_plan(dt)
    assert all(v == "filter" for v, _ in before)
    t_default = _time_steps(s, torch.from_numpy(C0).cuda(), dt)
    seg = s.autotune(dt)
    assert seg in (64, 96, 128, 192, 256, 384, 512)
    after = s.sweep_plan(dt)
    assert all(v == "filter" for v, _ in after)
    t_tuned = _time_steps(s, torch.from_numpy(C0).cuda(), dt)
    assert t_tuned <= 1.10 * t_default, (before, after, t_default, t_tuned)
    # parity of the tuned geometry with the oracle
    ref = oracle.run(oracle.grid(N, bc=1, vel=2, vp=(2 * np.pi, 0.5, 0.5), K=K,
                                 threads=THREADS, scheme=1), C0, 0.0, dt, 2)
    c = torch.from_numpy(C0).cuda()
    s.run(c, 0.0, dt, 2)
    s.check()
    assert rel_l2(c.cpu().numpy(), ref) < 1e-12
