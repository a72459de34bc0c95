"""The C-ABI library loads and exports every symbol include/ccfv.h declares;
argument validation needs no GPU."""
import ctypes as C

import pytest


def test_library_exports_every_declared_symbol(ccfv):
    names = ccfv.header_functions()
    assert len(names) >= 10
    L = ccfv.lib()
    for n in names:
        assert hasattr(L, n), n
    # every declared function has a ctypes signature in the binding
    assert set(names) <= set(ccfv._SIGS)


def test_strerror_covers_all_codes(ccfv):
    L = ccfv.lib()
    for code in range(10):
        assert L.ccfv_strerror(code).decode() != "unknown status"
    assert L.ccfv_strerror(999).decode() == "unknown status"


@pytest.mark.parametrize("mutate", [
    lambda g: setattr(g, "nx", 2),
    lambda g: setattr(g, "x_max", -5.0),
    lambda g: setattr(g, "bc", 7),
    lambda g: setattr(g, "velocity", 9),
    lambda g: setattr(g, "K", -1.0),
    lambda g: setattr(g, "scheme", 3),
])
def test_create_rejects_invalid_grid(ccfv, mutate):
    g = ccfv.make_grid(32, K=1e-3)
    mutate(g)
    h = C.c_void_p()
    rc = ccfv.lib().ccfv_create(C.byref(h), C.byref(g), 0)
    assert rc == ccfv.ERR_INVALID
    assert not h.value


def test_null_arguments_rejected(ccfv):
    L = ccfv.lib()
    assert L.ccfv_step(None, None, 0.0, 0.1, None) == ccfv.ERR_INVALID
    assert L.ccfv_destroy(None) == ccfv.ERR_INVALID
    assert L.ccfv_parareal(None, None, None, None, None, None) == ccfv.ERR_INVALID


def test_coarse_theta_resolves_like_the_oracle_rule(ccfv, oracle):
    """ccfv_coarse_theta (host only): 0 -> 0.5, fixed weights pass through,
    the automatic weight equals the oracle's restatement of the rule for
    coarse steps of (t1 - t0) / n_slices / m, and invalid weights are
    rejected."""
    kw = dict(t0=0.0, t1=1.0, nt_fine=512, n_slices=64, coarse_ratio=8)
    g = ccfv.make_grid(128, bc=ccfv.BC_PERIODIC, velocity=ccfv.VEL_CONST, vel_params=(1.0, 0.5),
                       K=0.01, scheme=ccfv.SCHEME_CONSISTENT)
    assert ccfv.coarse_theta(g, coarse_theta=0.0, **kw) == 0.5
    assert ccfv.coarse_theta(g, coarse_theta=0.8, **kw) == 0.8
    for bad in (0.3, 1.2, -2.0):
        with pytest.raises(ccfv.CcfvError):
            ccfv.coarse_theta(g, coarse_theta=bad, **kw)
    for nx, ny, K, ratio, dom in [(128, 128, 0.01, 8, None), (200, 96, 0.1, 4, None),
                                  (64, 64, 1e-4, 8, None), (300, 300, 0.05, 2, None),
                                  (100, 150, 0.2, 8, (0.0, 2.0, 0.0, 1.0))]:
        g = ccfv.make_grid(nx, ny, bc=ccfv.BC_PERIODIC, velocity=ccfv.VEL_CONST,
                           vel_params=(1.0, 0.5), K=K, domain=dom,
                           scheme=ccfv.SCHEME_CONSISTENT)
        o = oracle.grid(nx, ny, bc=oracle.BC_PERIODIC, vel=oracle.VEL_CONST, vp=(1.0, 0.5), K=K,
                        domain=dom, scheme=1)
        k2 = dict(kw, coarse_ratio=ratio)
        th = ccfv.coarse_theta(g, coarse_theta=ccfv.COARSE_THETA_AUTO, **k2)
        dtc = (k2["t1"] - k2["t0"]) / k2["n_slices"] / ((k2["nt_fine"] // k2["n_slices"]) // ratio)
        assert th == pytest.approx(oracle.auto_theta(o, dtc), rel=1e-14, abs=1e-15)
        assert 0.5 <= th <= 1.0
