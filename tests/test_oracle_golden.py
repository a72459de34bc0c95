"""The oracle against golden vectors produced by the reference itself.

tests/golden/*.npz were written by tests/golden/make_golden.py, which runs
the reference T2S4_Parareal.cu (compiled from its own source) on a B200.
These tests pin the CPU oracle; the CUDA path is then checked against it.
"""
import glob
import json
from pathlib import Path

import numpy as np
import pytest

from conftest import rel_l2

GOLDEN = sorted(glob.glob(str(Path(__file__).parent / "golden" / "*.npz")))
TOL = 1e-12  # relative L2, FP64 (parity bar for the fine result)


def _load(f):
    z = np.load(f)
    return json.loads(str(z["meta"])), z


@pytest.mark.parametrize("f", [g for g in GOLDEN if _load(g)[0]["kind"] in ("run", "ic_run")],
                         ids=lambda p: Path(p).stem)
def test_oracle_matches_reference_run(oracle, f):
    meta, z = _load(f)
    g = oracle.grid(meta["N"], K=meta["K"])
    out = oracle.run(g, z["C0"], meta["t0"], meta["dt"], meta["nsteps"])
    assert rel_l2(out, z["out"]) < TOL


def test_oracle_initial_condition_matches_reference(oracle):
    meta, z = _load(str(Path(__file__).parent / "golden" / "ic_N64.npz"))
    g = oracle.grid(meta["N"], K=meta["K"])
    assert rel_l2(oracle.exact_ref(g, 0.0), z["C0"]) < 1e-15
    assert rel_l2(oracle.exact_ref(g, meta["T"]), z["exact_T"]) < 1e-15


def test_oracle_parareal_schedule_matches_reference(oracle):
    meta, z = _load(str(Path(__file__).parent / "golden" / "parareal_N24.npz"))
    g = oracle.grid(meta["N"], K=meta["K"])
    uref = oracle.run(g, z["C0"], 0.0, meta["T_max"] / meta["Nt"], meta["Nt"])
    assert rel_l2(uref, z["uref"]) < TOL
    UT, err = oracle.parareal_ref(g, z["C0"], meta["T_min"], meta["T_max"], meta["Nt"],
                                  meta["n_slices"], meta["kmax"], Uref=uref)
    assert rel_l2(UT, z["UT"]) < TOL
    np.testing.assert_allclose(err, z["err"], rtol=1e-9, atol=1e-15)


def test_planted_mistake_is_caught(oracle):
    """A deliberately wrong oracle (the reference's third-sweep derivative
    rule switched off) must fail the golden comparison: the pin is sharp."""
    meta, z = _load(str(Path(__file__).parent / "golden" / "run_N32.npz"))
    g = oracle.grid(meta["N"], K=meta["K"], scheme=oracle.SCHEME_CONSISTENT)
    out = oracle.run(g, z["C0"], meta["t0"], meta["dt"], meta["nsteps"])
    assert rel_l2(out, z["out"]) > 1e-9
