"""CUDA path against the reference itself (oracle/_ref/libt2s4ref.so, built
from the reference source by `make -C oracle ref`), at sizes larger than the
committed golden vectors.  Skipped where that library is absent."""
import numpy as np
import pytest

from conftest import rel_l2, seeded_field

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def refh(oracle):
    if not oracle.ref_available():
        pytest.skip("reference harness not built")
    return oracle


@pytest.mark.parametrize("N,K,steps", [(128, 1e-3, 10), (256, 5e-4, 5), (512, 1e-4, 2)])
def test_cuda_matches_reference_binary(refh, ccfv, N, K, steps):
    import torch
    C0 = seeded_field(N, 100 + N)
    dt = 0.5 * (2.0 / N) / 4.0
    ref = refh.ref_run(N, K, 0.0, dt, steps, C0)
    s = ccfv.Solver(ccfv.make_grid(N, K=K))
    c = torch.from_numpy(C0).cuda()
    s.run(c, 0.0, dt, steps)
    s.check()
    assert rel_l2(c.cpu().numpy(), ref) < 1e-12


def test_reference_ic_matches_oracle(refh):
    g = refh.grid(96, K=1e-3)
    assert rel_l2(refh.exact_ref(g, 0.2), refh.ref_exact(96, 1e-3, 0.2)) < 1e-15
