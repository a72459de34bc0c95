"""Failure paths, made on the host (no device fault is ever provoked):

* invalid Parareal options are refused with CCFV_ERR_INVALID before any
  device work (the reference silently truncates J = Nt / 40 and runs
  whatever it gets, T2S4_Parareal.cu:1252);
* an allocation failure of the HBM-budget allocator, injected through
  CCFV_INJECT_ALLOC_FAIL (the k-th problem allocation of an engine reports
  an allocation failure instead of allocating): a batch returns
  CCFV_ERR_NOMEM and the library stays usable; in the server only the
  request whose allocation failed fails, the others complete with the same
  results as alone.
"""
import os

import numpy as np
import pytest

from conftest import periodic_field, rel_l2

pytestmark = pytest.mark.gpu


def _grid(ccfv, N=64):
    return ccfv.make_grid(N, bc=ccfv.BC_PERIODIC, velocity=ccfv.VEL_CONST,
                          vel_params=(1.0, -0.5), K=1e-3, scheme=ccfv.SCHEME_CONSISTENT)


GOOD = dict(t0=0.0, t1=0.25, nt_fine=64, n_slices=8, coarse_ratio=2, tol=0.0, kmax=3,
            coarse_precision=0, form=1)
BAD = [
    ("nt_not_multiple_of_slices", dict(nt_fine=65)),
    ("fewer_steps_than_slices", dict(nt_fine=4)),
    ("ratio_not_dividing", dict(coarse_ratio=3)),
    ("kmax_zero", dict(kmax=0)),
    ("kmax_too_large", dict(kmax=1000)),
    ("fp32_standard_form", dict(coarse_precision=1, form=0)),
    ("unknown_form", dict(form=7)),
    ("theta_out_of_range", dict(coarse_theta=0.3)),
]


@pytest.mark.parametrize("name,bad", BAD, ids=[b[0] for b in BAD])
def test_invalid_parareal_options_rejected(ccfv, name, bad):
    import torch
    s = ccfv.Solver(_grid(ccfv))
    C0 = torch.from_numpy(periodic_field(64, 1)).cuda()
    out = torch.full_like(C0, 7.0)
    kw = dict(GOOD, **bad)
    with pytest.raises(ccfv.CcfvError) as ei:
        s.parareal(C0, out, **kw)
    assert ei.value.status == ccfv.ERR_INVALID
    assert float(out.min()) == 7.0 == float(out.max())  # nothing written
    # the same options in a batch
    with pytest.raises(ccfv.CcfvError) as ei:
        ccfv.batch_solve([dict(kw, grid=_grid(ccfv), C0=C0, C_T=out)])
    assert ei.value.status == ccfv.ERR_INVALID


def _problems(ccfv, n):
    import torch
    probs = []
    for i in range(n):
        N = 48 + 16 * i
        C0 = torch.from_numpy(periodic_field(N, 10 + i)).cuda()
        probs.append(dict(GOOD, grid=_grid(ccfv, N), C0=C0, C_T=torch.empty_like(C0),
                          coarse_precision=1))
    return probs


def test_batch_allocation_failure_is_reported_and_recovers(ccfv, monkeypatch):
    probs = _problems(ccfv, 4)
    monkeypatch.setenv("CCFV_INJECT_ALLOC_FAIL", "3")
    with pytest.raises(ccfv.CcfvError) as ei:
        ccfv.batch_solve(probs)
    assert ei.value.status == ccfv.ERR_NOMEM
    monkeypatch.delenv("CCFV_INJECT_ALLOC_FAIL")
    st = ccfv.batch_solve(probs)
    for p, x in zip(probs, st):
        s = ccfv.Solver(p["grid"])
        kw = {k: p[k] for k in GOOD}
        ref, _ = s.parareal(p["C0"], **kw)
        assert x["iterations"] == 3
        assert rel_l2(p["C_T"].cpu().numpy(), ref.cpu().numpy()) < 1e-12


def test_server_allocation_failure_fails_only_that_request(ccfv, monkeypatch):
    probs = []
    for i in range(3):
        N = 64 + 32 * i
        C0 = periodic_field(N, 20 + i)
        probs.append(dict(GOOD, grid=_grid(ccfv, N), C0=C0, C_T=np.empty_like(C0),
                          coarse_precision=1))
    refs = []
    for p in probs:
        s = ccfv.Solver(p["grid"])
        refs.append(s.parareal(p["C0"], **{k: p[k] for k in GOOD})[0])
    monkeypatch.setenv("CCFV_INJECT_ALLOC_FAIL", "2")
    srv = ccfv.Server(hbm_budget_bytes=1 << 30, max_active=1)  # admitted one by one
    try:
        tickets = [srv.submit(p) for p in probs]
        outcome = []
        for t in tickets:
            try:
                srv.wait(t, timeout_s=60.0)
                outcome.append(ccfv.OK)
            except ccfv.CcfvError as e:
                outcome.append(e.status)
    finally:
        srv.close()
        os.environ.pop("CCFV_INJECT_ALLOC_FAIL", None)
    assert outcome == [ccfv.OK, ccfv.ERR_NOMEM, ccfv.OK]
    for i in (0, 2):
        assert rel_l2(probs[i]["C_T"], refs[i]) < 1e-12
