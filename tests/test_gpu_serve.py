"""Serving loop (ccfv_server_*): continuous batching with HBM-budget
admission.  Each result is the same alone and in the mix (FP64 parity
tolerance), requests that arrive while others run are admitted and overlap,
oversize requests are rejected, queued requests can be cancelled."""
import time

import numpy as np
import pytest

from conftest import periodic_field, rel_l2

pytestmark = pytest.mark.gpu


def _req(ccfv, N, vel, vp, K, seed, T=0.25, S=8, ratio=2, prec=1, tol=1e-10):
    g = ccfv.make_grid(N, bc=1, velocity=vel, vel_params=vp, K=K, scheme=1)
    C0 = periodic_field(N, seed)
    nt = 8 * S
    return dict(grid=g, C0=C0, C_T=np.empty_like(C0), t0=0.0, t1=T, nt_fine=nt, n_slices=S,
                coarse_ratio=ratio, tol=tol, kmax=S, coarse_precision=prec, form=1)


def _alone(ccfv, p):
    s = ccfv.Solver(p["grid"])
    out, st = s.parareal(p["C0"], t0=p["t0"], t1=p["t1"], nt_fine=p["nt_fine"],
                         n_slices=p["n_slices"], coarse_ratio=p["coarse_ratio"], tol=p["tol"],
                         kmax=p["kmax"], coarse_precision=p["coarse_precision"], form=p["form"])
    return out, st


MIX = [(96, 1, (1.0, -0.4), 1e-3), (160, 2, (2 * np.pi, 0.5, 0.5), 1e-3),
       (64, 3, (1.5,), 5e-4), (300, 1, (-0.3, 0.8), 1e-4), (128, 2, (2 * np.pi, 0.5, 0.5), 1e-2)]


# long enough (tens of milliseconds) that requests submitted once they run
# are admitted while they still run
EARLY = [(400, 2, (2 * np.pi, 0.5, 0.5), 1e-3), (512, 1, (1.0, -0.4), 1e-3)]


def test_server_results_equal_alone_and_late_arrivals_overlap(ccfv):
    reqs = [_req(ccfv, N, v, vp, K, i, S=16) for i, (N, v, vp, K) in enumerate(EARLY)]
    reqs += [_req(ccfv, N, v, vp, K, i) for i, (N, v, vp, K) in enumerate(MIX[2:], start=2)]
    refs = [_alone(ccfv, p) for p in reqs]
    srv = ccfv.Server(hbm_budget_bytes=8 << 30)
    try:
        tickets = [srv.submit(p) for p in reqs[:2]]
        # wait until the first requests are resident, then submit the rest
        t0 = time.time()
        while srv.poll(tickets[0])[1] == ccfv.REQ_QUEUED and time.time() - t0 < 30:
            time.sleep(0.001)
        late = [srv.submit(p) for p in reqs[2:]]
        overlapped = False
        t0 = time.time()
        while time.time() - t0 < 60:
            st_early = [srv.poll(t)[1] for t in tickets]
            st_late = [srv.poll(t)[1] for t in late]
            if ccfv.REQ_RUNNING in st_early and ccfv.REQ_RUNNING in st_late:
                overlapped = True
            if all(s == ccfv.REQ_DONE for s in st_early + st_late):
                break
            time.sleep(0.0005)
        results = [srv.wait(t, timeout_s=120) for t in tickets + late]
    finally:
        srv.close()
    for p, (ref, st_a), (st_b, lat) in zip(reqs, refs, results):
        assert st_b["iterations"] == st_a["iterations"]
        assert rel_l2(p["C_T"], ref) < 1e-12
        assert lat > 0
    assert overlapped, "late requests never ran alongside the early ones"


def test_server_budget_admission_and_rejection(ccfv):
    small = _req(ccfv, 64, 1, (1.0, 0.5), 1e-3, 1)
    # slice states U and F, F's out-of-place partner (S fields), and the coarse
    # work field and its partner (FP64-sized: the first coarse sweep is FP64)
    S = small["n_slices"]
    need = (2 * (S + 1) + S + 2) * 64 * 64 * 8 + 4096
    srv = ccfv.Server(hbm_budget_bytes=need)  # room for exactly one resident request
    try:
        big = _req(ccfv, 256, 1, (1.0, 0.5), 1e-3, 2)
        with pytest.raises(ccfv.CcfvError) as ei:
            srv.submit(big)
        assert ei.value.status == ccfv.ERR_BUDGET
        reqs = [_req(ccfv, 64, 1, (1.0, 0.5), 1e-3, s) for s in range(3)]
        ts = [srv.submit(p) for p in reqs]
        for t in ts:
            st, _ = srv.wait(t, timeout_s=60)
            assert st["iterations"] >= 1
        assert srv.info()["used_bytes"] == 0
    finally:
        srv.close()
    for p in reqs:
        ref, _ = _alone(ccfv, p)
        assert rel_l2(p["C_T"], ref) < 1e-12


def test_server_cancel_queued(ccfv):
    srv = ccfv.Server(hbm_budget_bytes=1 << 28, max_active=1)
    try:
        first = srv.submit(_req(ccfv, 256, 2, (2 * np.pi, 0.5, 0.5), 1e-3, 1, S=16))
        second = srv.submit(_req(ccfv, 64, 1, (1.0, 0.5), 1e-3, 2))
        assert srv.cancel(second) == 0
        with pytest.raises(ccfv.CcfvError) as ei:
            srv.wait(second, timeout_s=60)
        assert ei.value.status == ccfv.ERR_CANCELLED
        st, _ = srv.wait(first, timeout_s=120)
        assert st["iterations"] >= 1
    finally:
        srv.close()
