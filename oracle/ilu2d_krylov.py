"""What a 2D block ILU(0) preconditioner would save: GMRES(20) iteration counts of the first
backward-Euler Newton solve (CFL 5, the rotated simple wave, ltol 1e-12) with block-Jacobi (the
reference's only 2D preconditioner) and with block ILU(0) in the natural ordering on the
cartesian block graph (the oracle's BlockILU0 restatement of block_ilu.cpp), both on the
oracle's DG Jacobian.  CPU only; the oracle is the reference's algorithm restated, so this
measures the preconditioners, not this repository's kernels.

    python oracle/ilu2d_krylov.py [--cases 16x2,32x2,16x4,32x4,8x8,16x8,32x8]

Per case it prints the two Krylov counts, their ratio and the two refresh times of the oracle
(single-threaded dense loops: their ratio approximates the flop ratio of the factorisations).
"""
from __future__ import annotations

import argparse
import sys
import time
from pathlib import Path

sys.path.insert(0, str(Path(__file__).resolve().parent))

import oracle_py  # noqa: E402


def case(nx: int, k: int, cfl: float = 5.0, restart: int = 20, tol: float = 1e-12) -> dict:
    o = oracle_py.Oracle(f"--nx {nx} --ny {nx} --k {k} --cfl {cfl} --integrator be --steps 1 --restart {restart}")
    u = o.initial()
    dt = cfl / o.freeze(u)
    o.set_stage(u, dt)
    r = o.residual(u)
    o.dg_refresh(u)
    out = {"nx": nx, "k": k, "m": o.block}
    t = time.perf_counter()
    o.dg_precond_refresh()
    out["bj_refresh_s"] = time.perf_counter() - t
    _, out["bj_krylov"], out["bj_rel"], _ = o.gmres(0, -r, restart, 5000, tol)
    t = time.perf_counter()
    o.dg_precond_refresh_ilu()
    out["ilu_refresh_s"] = time.perf_counter() - t
    _, out["ilu_krylov"], out["ilu_rel"], _ = o.gmres(2, -r, restart, 5000, tol)
    return out


def main(argv=None) -> None:
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--cases", default="16x2,32x2,16x4,32x4,8x8,16x8,32x8")
    a = ap.parse_args(argv)
    print("| mesh | k | block-Jacobi Krylov | block ILU(0) Krylov | ratio | refresh s (BJ / ILU) |")
    print("|---|---|---|---|---|---|")
    for c in a.cases.split(","):
        nx, k = (int(v) for v in c.split("x"))
        d = case(nx, k)
        print(f"| {nx}² | {k} | {d['bj_krylov']} | {d['ilu_krylov']} | {d['bj_krylov'] / max(d['ilu_krylov'], 1):.2f} | "
              f"{d['bj_refresh_s']:.2f} / {d['ilu_refresh_s']:.2f} |", flush=True)


if __name__ == "__main__":
    main()
