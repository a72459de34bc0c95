"""ccfv_step_noalloc: the split step for callers that cannot allocate device
memory (its scratch is a fixed device array inside the library).  Checked
through the C ABI against ccfv_step on two calls in a row.  This file is
collected last so that a failure here stops a `-x` run only after every other
test has run."""
import ctypes as C

import numpy as np
import pytest

from conftest import periodic_field, rel_l2, seeded_field

pytestmark = pytest.mark.gpu

CASES = [
    ("compat_reference", dict(bc=0, velocity=0, K=1e-3, scheme=0), 96, 96, 0.004),
    ("periodic_rotation_cluster", dict(bc=1, velocity=2, vel_params=(2 * np.pi, 0.5, 0.5),
                                       K=1e-3, scheme=1), 300, 260, 0.8 / 300 / np.pi),
    ("periodic_swirl", dict(bc=1, velocity=3, vel_params=(1.5,), K=5e-4, scheme=1), 128, 128,
     0.005),
    ("compat_gaussian_source", dict(bc=0, velocity=0, K=1e-3, scheme=0, source=1,
                                    source_params=(2.0, 0.2, -0.1, 0.05, 3.0)), 80, 72, 0.004),
    ("periodic_gaussian_source", dict(bc=1, velocity=2, vel_params=(2 * np.pi, 0.5, 0.5),
                                      K=1e-3, scheme=1, source=1,
                                      source_params=(1.5, 0.4, 0.6, 0.02, 5.0)), 96, 96, 0.002),
]


@pytest.mark.parametrize("name,kw,nx,ny,dt", CASES, ids=[c[0] for c in CASES])
def test_step_noalloc_matches_step(ccfv, name, kw, nx, ny, dt):
    import torch
    grid = ccfv.make_grid(nx, ny, **kw)
    C0 = seeded_field(nx, 5, ny=ny) if kw["bc"] == 0 else periodic_field(nx, 5, ny=ny)
    a = torch.from_numpy(C0).cuda()
    b = torch.from_numpy(C0).cuda()
    s = ccfv.Solver(grid)
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    for call in range(2):  # two calls in a row share the static scratch
        tn = 0.1 + call * dt
        s.step(a, tn, dt)
        torch.cuda.synchronize()
        free0 = torch.cuda.mem_get_info()[0]
        rc = ccfv.lib().ccfv_step_noalloc(C.byref(grid), C.c_void_p(b.data_ptr()), tn, dt,
                                          stream)
        assert rc == ccfv.OK, ccfv.lib().ccfv_strerror(rc)
        torch.cuda.synchronize()
        if call == 1:  # after a warm-up call (lazy module loading): no device memory taken
            assert torch.cuda.mem_get_info()[0] == free0, name
        assert rel_l2(b.cpu().numpy(), a.cpu().numpy()) < 1e-12, (name, call)


def test_step_noalloc_rejects_oversize_grid(ccfv):
    import torch
    grid = ccfv.make_grid(4097, 64, K=1e-3)
    buf = torch.zeros(4097 * 64, dtype=torch.float64, device="cuda")
    rc = ccfv.lib().ccfv_step_noalloc(C.byref(grid), C.c_void_p(buf.data_ptr()), 0.0, 1e-3, None)
    assert rc == ccfv.ERR_UNSUPPORTED


def test_step_noalloc_rejects_oversize_time_step(ccfv):
    """A time step whose characteristic shift does not fit the staged halo in
    shared memory is refused on the host, before any device work."""
    import torch
    N = 64
    grid = ccfv.make_grid(N, bc=1, velocity=1, vel_params=(1.0, 1.0), K=1e-3, scheme=1)
    buf = torch.zeros(N * N, dtype=torch.float64, device="cuda")
    rc = ccfv.lib().ccfv_step_noalloc(C.byref(grid), C.c_void_p(buf.data_ptr()), 0.0, 20.0, None)
    assert rc == ccfv.ERR_UNSUPPORTED
    assert float(buf.abs().sum()) == 0.0
