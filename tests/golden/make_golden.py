"""Generate golden vectors by running the reference itself.

Runs the reference T2S4_Parareal.cu (compiled from its own source into
oracle/_ref/libt2s4ref.so by `make -C oracle ref`) on seeded inputs and
saves full-FP64 inputs and outputs as .npz fixtures.  Needs a GPU.

    python tests/golden/make_golden.py [outdir]

The fixtures are committed under tests/golden/ and pin the CPU oracle
(tests/test_oracle_golden.py) and the CUDA path (tests/test_gpu_parity.py).
"""
from __future__ import annotations

import json
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT / "oracle"))
import oracle as O  # noqa: E402


def seeded_field(N: int, seed: int) -> np.ndarray:
    """Smooth random field on [-1,1]^2, non-zero on the boundary, plus noise."""
    rng = np.random.default_rng(seed)
    x = -1.0 + (np.arange(N) + 0.5) * (2.0 / N)
    X, Y = np.meshgrid(x, x, indexing="ij")
    f = 0.2 + 0.1 * X - 0.05 * Y
    for _ in range(4):
        cx, cy = rng.uniform(-0.8, 0.8, 2)
        w = rng.uniform(0.05, 0.3)
        a = rng.uniform(0.3, 1.0)
        f = f + a * np.exp(-((X - cx) ** 2 + (Y - cy) ** 2) / w)
    f = f + 1e-3 * rng.standard_normal((N, N))
    return np.ascontiguousarray(f)


CASES = [
    # name, N, K, t0, dt, nsteps, seed
    ("step_N16", 16, 1e-3, 0.0, 0.01, 1, 101),
    ("run_N32", 32, 5e-3, 0.0, 2e-3, 10, 102),
    ("run_N48", 48, 1e-2, 0.1, 5e-3, 5, 103),
    ("bigcfl_N32", 32, 0.05, 0.0, 0.05, 3, 104),
    ("run_N64", 64, 1e-3, 0.0, 2.5e-3, 20, 105),
]


def main(outdir: Path) -> None:
    outdir.mkdir(parents=True, exist_ok=True)
    for name, N, K, t0, dt, nsteps, seed in CASES:
        C0 = seeded_field(N, seed)
        out = O.ref_run(N, K, t0, dt, nsteps, C0)
        meta = dict(kind="run", N=N, K=K, t0=t0, dt=dt, nsteps=nsteps, seed=seed)
        np.savez_compressed(outdir / f"{name}.npz", meta=json.dumps(meta), C0=C0, out=out)
        print(name, "ok", float(np.abs(out).max()))
    # the reference's own initial condition run (T2S4_Parareal.cu:1147-1161, 1234-1247)
    N, K, T, Nt = 64, 1e-3, 0.1, 40
    ic = O.ref_exact(N, K, 0.0)
    ex = O.ref_exact(N, K, T)
    out = O.ref_run(N, K, 0.0, T / Nt, Nt, ic)
    meta = dict(kind="ic_run", N=N, K=K, t0=0.0, dt=T / Nt, nsteps=Nt, T=T)
    np.savez_compressed(outdir / "ic_N64.npz", meta=json.dumps(meta), C0=ic, out=out, exact_T=ex)
    print("ic_N64 ok")
    # Parareal schedule (T2S4_Parareal.cu:1249-1355), 40 slices, small grid
    N, K, T, Nt, S, kmax = 24, 2e-3, 0.2, 80, 40, 3
    C0 = seeded_field(N, 106)
    uref = O.ref_run(N, K, 0.0, T / Nt, Nt, C0)
    UT, err = O.ref_parareal(N, K, 0.0, T, Nt, C0, n_slices=S, kmax=kmax, Uref=uref)
    meta = dict(kind="parareal", N=N, K=K, T_min=0.0, T_max=T, Nt=Nt, n_slices=S, kmax=kmax,
                seed=106)
    np.savez_compressed(outdir / "parareal_N24.npz", meta=json.dumps(meta), C0=C0, uref=uref,
                        UT=UT, err=err)
    print("parareal_N24 ok", err)


if __name__ == "__main__":
    main(Path(sys.argv[1]) if len(sys.argv) > 1 else Path(__file__).resolve().parent)
