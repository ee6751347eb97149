"""Generates tests/golden/*.npz from the reference's own CUDA kernels.

Runs where a GPU and oracle/_ref/libpicref.so (built by `make -C oracle ref` from the
reference's sources) are available:  python tests/golden/make_golden.py [outdir] [--only embedded]
Every fixture stores its seeded inputs and the reference's outputs; tests/test_golden.py
checks that the FP64 oracle reproduces them (CPU only).
"""
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from oracle import refh  # noqa: E402

Q, M = [0.1, -1.0], [1.0, 1.0]
WALLS = [[0, 0, 1, 0], [1, 0, 1, 1], [1, 1, 0, 1], [0, 1, 0, 0], [0.25, 0.25, 0.25, 0.75], [0.75, 0.25, 0.75, 0.75]]


def main(out: Path, only: str | None = None):
    out.mkdir(parents=True, exist_ok=True)
    assert refh.available(), "needs a GPU and oracle/_ref/libpicref.so"
    if only in (None, "embedded"):
        embedded(out)
    if only == "embedded":
        return
    rng = np.random.default_rng(20240601)
    # updateDensity (kernels.cu:26)
    n = 4000
    x, y = rng.random(n), rng.random(n)
    t = rng.integers(0, 2, n).astype(np.int32)
    rho = refh.deposit(x, y, t, Q, 65, 65, 1 / 64, 1 / 64)
    np.savez_compressed(out / "ref_deposit.npz", x=x, y=y, type=t, q=np.array(Q), m=65, n=65, dx=1 / 64, rho=rho)
    # solve_multigrid (Multigrid.cu:573), the reference's own call shape (5 levels, omega 1.25)
    for nn, lev in ((65, 4), (129, 5)):
        f = rng.standard_normal((nn, nn))
        phi0 = np.zeros((nn, nn))
        phi0[0, :] = 0.25
        phi = refh.solve(phi0, f, 1.0 / (nn - 1), levels=lev, omega=1.25)
        np.savez_compressed(out / f"ref_solve_{nn}.npz", f=f, phi0=phi0, phi=phi, levels=lev, h=1.0 / (nn - 1))
    # computeElectricField (kernels.cu:134)
    phi = rng.standard_normal((33, 65))
    ex, ey = refh.efield(phi, 0.1, 0.2)
    np.savez_compressed(out / "ref_efield.npz", phi=phi, ex=ex, ey=ey, dx=0.1, dy=0.2)
    # one re-sequenced updateSimulationCUDA step (main.cu:60-135) on 65^2, walls of main.cu:193-194 + box
    n = 4000
    x, y = rng.random(n) * 0.98 + 0.01, rng.random(n) * 0.98 + 0.01
    vx, vy = rng.uniform(-1, 1, n), rng.uniform(-1, 1, n)
    t = rng.integers(0, 2, n).astype(np.int32)
    dt = 0.01
    from oracle import oracle as o
    hit = o.walls_segments(x, y, x + vx * dt, y + vy * dt, WALLS)
    order = np.concatenate([np.nonzero(hit)[0], np.nonzero(~hit)[0]])  # no tail hits, <= 256 holes
    x, y, vx, vy, t = x[order], y[order], vx[order], vy[order], t[order]
    r = refh.steps(1, x, y, vx, vy, t, Q, M, 65, 65, 1.0, 1.0, WALLS, dt)
    np.savez_compressed(out / "ref_step.npz", x=x, y=y, vx=vx, vy=vy, type=t, q=np.array(Q), mass=np.array(M),
                        walls=np.array(WALLS, float), dt=dt, m=65, n=65, x1=r["x"], y1=r["y"], vx1=r["vx"],
                        vy1=r["vy"], type1=r["type"], rho1=r["rho"], phi1=r["phi"], hits=np.sort(r["hits"]))
    print("wrote", sorted(p.name for p in out.glob("*.npz")))


def embedded(out: Path):
    """The kernels of Multigrid_embedded.cu on a rectangular level with an electrode whose
    edges sit on odd and even node indices and a solid block (own seed)."""
    rng = np.random.default_rng(20241203)
    nx, ny = 65, 49
    mask = np.zeros((ny, nx), np.uint8)
    mask[12:25, 16:31] = 1
    mask[30:41, 40:52] = 2
    bc = np.zeros((ny, nx))
    bc[mask == 1] = 2.5
    phi = rng.standard_normal((ny, nx))
    rhs = rng.standard_normal((ny, nx))
    h2 = (1.0 / 64) ** 2
    phi_c = rng.standard_normal(((ny - 1) // 2 + 1, (nx - 1) // 2 + 1))
    r = refh.emb_kernels(phi, rhs, mask, bc, h2, phi_c)
    np.savez_compressed(out / "ref_embedded.npz", phi=phi, rhs=rhs, mask=mask, bc=bc, h2=h2, phi_c=phi_c, **r)


if __name__ == "__main__":
    import argparse
    ap = argparse.ArgumentParser()
    ap.add_argument("outdir", nargs="?", default=str(Path(__file__).resolve().parent))
    ap.add_argument("--only", choices=["embedded"], default=None, help="write only this fixture")
    a = ap.parse_args()
    main(Path(a.outdir), a.only)
