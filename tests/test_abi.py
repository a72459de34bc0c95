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
