"""How the storage precision of the block-Jacobi factors changes the GMRES(20) iteration count
of the first backward-Euler Newton solve (CFL 5, the rotated simple wave, tolerance 1e-12 in the
inverse-mass-weighted norm), on the oracle's DG Jacobian.  Each cell block is factored with row
partial pivoting in FP64 (scipy's getrf), the packed L\\U factors are rounded to fp64, fp32,
fp16 or bf16 (round to nearest even), and the preconditioner solves with the rounded factors.
CPU only; a sizing experiment for the factor stream, which dominates the device's DG update.

    python oracle/factor_precision_krylov.py [--cases 8x4,8x8,16x8]
"""
from __future__ import annotations

import argparse
import sys
from pathlib import Path

import numpy as np
import scipy.linalg as sl

sys.path.insert(0, str(Path(__file__).resolve().parent))

import oracle_py  # noqa: E402

KINDS = ("fp64", "fp32", "fp16", "bf16")


def rounded(a: np.ndarray, kind: str) -> np.ndarray:
    if kind == "fp64":
        return a
    if kind == "fp32":
        return a.astype(np.float32).astype(np.float64)
    if kind == "fp16":
        return a.astype(np.float16).astype(np.float64)
    bits = a.astype(np.float32).view(np.uint32)  # bf16: keep the upper 16 bits, rounded to nearest even
    bits = ((bits + np.uint32(0x7FFF) + ((bits >> np.uint32(16)) & np.uint32(1))) & np.uint32(0xFFFF0000))
    return bits.astype(np.uint32).view(np.float32).astype(np.float64)


def gmres(apply_a, apply_m, b, weights, restart=20, tol=1e-12, limit=5000):
    """Right-preconditioned restarted GMRES with classical Gram-Schmidt applied twice, in the
    weighted inner product; returns the iteration count at which the Arnoldi residual estimate
    reaches tol relative to b."""
    dot = lambda p, q: float(np.sum(p * q * weights))
    bnorm = np.sqrt(dot(b, b))
    x, its = np.zeros_like(b), 0
    while its < limit:
        r = b - apply_a(x)
        beta = np.sqrt(dot(r, r))
        if beta <= tol * bnorm:
            return its
        V, Z = [r / beta], []
        H = np.zeros((restart + 1, restart))
        g = np.zeros(restart + 1)
        g[0] = beta
        y = np.zeros(0)
        for j in range(restart):
            z = apply_m(V[j])
            Z.append(z)
            v = apply_a(z)
            for _ in range(2):
                for i in range(j + 1):
                    h = dot(V[i], v)
                    H[i, j] += h
                    v = v - h * V[i]
            H[j + 1, j] = np.sqrt(dot(v, v))
            V.append(v / H[j + 1, j])
            its += 1
            y = np.linalg.lstsq(H[:j + 2, :j + 1], g[:j + 2], rcond=None)[0]
            if np.linalg.norm(H[:j + 2, :j + 1] @ y - g[:j + 2]) <= tol * bnorm:
                break
        x = x + np.array(Z).T @ y
    return its


def case(nx: int, k: int) -> dict[str, int]:
    o = oracle_py.Oracle(f"--nx {nx} --ny {nx} --k {k} --cfl 5 --integrator be --steps 1 --restart 20")
    u = o.initial()
    o.set_stage(u, 5.0 / o.freeze(u))
    r = o.residual(u)
    o.dg_refresh(u)
    m, cells = o.block, o.cells
    factors = [sl.lu_factor(o.dg_block(c, c)) for c in range(cells)]
    out = {}
    for kind in KINDS:
        fk = [(rounded(lu, kind), piv) for lu, piv in factors]

        def apply_m(v, fk=fk):
            z = np.empty_like(v)
            for c in range(cells):
                z[c * m:(c + 1) * m] = sl.lu_solve(fk[c], v[c * m:(c + 1) * m])
            return z

        out[kind] = gmres(o.dg_apply, apply_m, -r, 1.0 / o.mass)
    return out


def main(argv=None) -> None:
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--cases", default="8x4,8x8,16x8")
    a = ap.parse_args(argv)
    print("| mesh | k | " + " | ".join(KINDS) + " |")
    print("|---|---|" + "---|" * len(KINDS))
    for c in a.cases.split(","):
        nx, k = (int(v) for v in c.split("x"))
        d = case(nx, k)
        print(f"| {nx}² | {k} | " + " | ".join(str(d[kind]) for kind in KINDS) + " |", flush=True)


if __name__ == "__main__":
    main()
