"""Device initial-condition / exact-solution / norm kernels and the CLI
driver against the oracle and the reference's output format."""
import os
import subprocess
from pathlib import Path

import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu
ROOT = Path(__file__).resolve().parents[1]


def test_exact_ref_matches_oracle_and_golden(oracle, ccfv):
    import torch
    z = np.load(ROOT / "tests" / "golden" / "ic_N64.npz")
    s = ccfv.Solver(ccfv.make_grid(64, K=1e-3))
    c = torch.empty(64, 64, dtype=torch.float64, device="cuda")
    s.exact_ref(c, 0.0)
    assert rel_l2(c.cpu().numpy(), z["C0"]) < 1e-14
    s.exact_ref(c, 0.1)
    assert rel_l2(c.cpu().numpy(), z["exact_T"]) < 1e-14


def test_gaussians_match_oracle(oracle, ccfv):
    import torch
    g = oracle.grid(96, 80, bc=1)
    par = [[0.3, 0.7, 0.01, 1.0], [0.8, 0.2, 0.005, 0.5]]
    ref = oracle.gaussians(g, [p[0] for p in par], [p[1] for p in par], [p[2] for p in par],
                           [p[3] for p in par], img=1)
    s = ccfv.Solver(ccfv.make_grid(96, 80, bc=1))
    c = torch.empty(96, 80, dtype=torch.float64, device="cuda")
    s.gaussians(c, par, images=1)
    assert rel_l2(c.cpu().numpy(), ref) < 1e-14


def test_error_norms(ccfv):
    import torch
    rng = np.random.default_rng(1)
    a, b = rng.standard_normal((70, 50)), rng.standard_normal((70, 50))
    s = ccfv.Solver(ccfv.make_grid(70, 50, bc=1))
    r, m = s.error_norms(torch.from_numpy(a).cuda(), torch.from_numpy(b).cuda())
    assert abs(r - np.linalg.norm(a - b) / np.linalg.norm(b)) < 1e-13
    assert m == np.abs(a - b).max()


def test_parareal_reference_diagnostic_matches_golden(ccfv):
    """Per-iteration max-norm error against the serial solution, computed on
    the device, equals the reference's printed diagnostic."""
    import json
    import torch
    z = np.load(ROOT / "tests" / "golden" / "parareal_N24.npz")
    meta = json.loads(str(z["meta"]))
    s = ccfv.Solver(ccfv.make_grid(meta["N"], K=meta["K"]))
    ref = torch.from_numpy(z["uref"]).cuda()
    _, st = s.parareal(torch.from_numpy(z["C0"]).cuda(), t0=meta["T_min"], t1=meta["T_max"],
                       nt_fine=meta["Nt"], n_slices=meta["n_slices"], kmax=meta["kmax"], ref=ref)
    np.testing.assert_allclose(st["err_max"], z["err"], rtol=1e-9, atol=1e-15)


def test_cli_driver_matches_reference_interface(tmp_path, oracle):
    exe = ROOT / "parareal-cc-cfv-split-gpu_b200" / "bin" / "t2s4_parareal"
    if not exe.exists():
        pytest.skip("driver not built")
    cfg = tmp_path / "config.txt"
    cfg.write_text("T_min:0\nT_max:0.1\nN:32\nNt:40\nT_span:20\nK:0.001\n")
    r = subprocess.run([str(exe), str(cfg)], cwd=tmp_path, capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0, r.stderr
    out = r.stdout
    assert "open config file ok" in out
    assert out.count("Parareal iter") == 8
    assert "Total time (including Parareal):" in out and "Nx:32" in out
    dumps = sorted(p.name for p in tmp_path.glob("data_T2S4_*.txt"))
    assert dumps == ["data_T2S4_000000.txt", "data_T2S4_000020.txt", "data_T2S4_000040.txt"]
    # the final dump equals the oracle's serial run to the dump's 4 digits
    g = oracle.grid(32, K=1e-3)
    ref = oracle.run(g, oracle.exact_ref(g, 0.0), 0.0, 0.1 / 40, 40)
    vals = np.loadtxt(tmp_path / "data_T2S4_000040.txt")[:, 2].reshape(32, 32)
    assert np.abs(vals - ref).max() <= 5e-5 * max(1.0, np.abs(ref).max())


def test_cli_driver_usage_message():
    exe = ROOT / "parareal-cc-cfv-split-gpu_b200" / "bin" / "t2s4_parareal"
    if not exe.exists():
        pytest.skip("driver not built")
    r = subprocess.run([str(exe)], capture_output=True, text=True)
    assert r.returncode == 1 and "please input config file name" in r.stdout
