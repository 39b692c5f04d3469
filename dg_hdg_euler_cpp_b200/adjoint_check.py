"""Gradient of the DIRK3 DG solve with respect to Fourier coefficients of the initial density.

    python -m dg_hdg_euler_cpp_b200.adjoint_check [--nx 128 --k 4 --steps 20 --every 5 --cfl 2]

Objective J = sum over nodes of M rho^2 after `steps` SSP-DIRK3 steps of the DG solve (the
rotated simple wave, gamma = 3, CFL-limited dt).  Parameters: 8 Fourier coefficients theta of
a density perturbation added to the projected initial state at the nodes,
rho_0 += sum_k theta_k cos/sin(2 pi m (x / lx + y / ly)) for m = 1..4: the modes along the
wave's direction of variation (the base state depends on x + y only, so modes with kx != ky are
orthogonal to it and have zero gradient by symmetry).  The gradient comes from one discrete-adjoint solve
(dgh_dirk3_adjoint: J^T GMRES per stage, checkpoints every `every` steps, recompute in between)
and is compared with central finite differences (step h) of the same trajectory with dt and the
frozen speeds replayed (dgh_dirk3_replay).  Prints one JSON line.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import time

import numpy as np

MODES = [(1, 1), (2, 2), (3, 3), (4, 4)]


def fourier_modes(s, nx: int, ny: int, k: int) -> np.ndarray:
    """Density-only nodal fields of the 8 modes (rows), in the solver's state layout."""
    n = k + 1
    x = np.zeros(n)
    s.lib.dgh_nodes(s.h, x.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), None)
    hx, hy, lx, ly = s.hx, s.hy, s.lx, s.ly
    cells = nx * ny
    cx = (np.arange(cells) % nx)[:, None, None]
    cy = (np.arange(cells) // nx)[:, None, None]
    X = -.5 * lx + hx * (cx + .5) + .5 * hx * x[None, None, :]  # x node index fastest
    Y = -.5 * ly + hy * (cy + .5) + .5 * hy * x[None, :, None]
    phis = []
    for mx, my in MODES:
        arg = 2 * np.pi * (mx * X / lx + my * Y / ly)
        for f in (np.cos, np.sin):
            field = np.zeros((cells, 4, n, n))
            field[:, 0] = np.broadcast_to(f(arg), (cells, n, n))
            phis.append(field.reshape(-1))
    return np.array(phis)


def gradient_check(nx: int = 128, k: int = 4, steps: int = 20, every: int = 5, cfl: float = 2.0, h: float = 1e-6,
                   amplitude: float = 0.02) -> dict:
    """Adjoint gradient of J with respect to the 8 Fourier coefficients against central finite
    differences of the replayed trajectory; returns the record main() prints."""
    from . import _lib
    from .solver import Integrator, Solver

    s = Solver(nx=nx, ny=nx, k=k, cfl=cfl, integrator="ssp-dirk3", steps=steps, method="dg", restart=20)
    s.gmres_graph(True)
    it = Integrator(s, "dg")
    try:
        u0 = s.initial().cpu().numpy()
        phis = amplitude * fourier_modes(s, nx, nx, k)
        grad = np.zeros(s.size)
        st = _lib.dgh_adjoint_stats()
        t0 = time.perf_counter()
        rc = s.lib.dgh_dirk3_adjoint(it.h, steps, every, u0.ctypes.data_as(ctypes.c_void_p),
                                     grad.ctypes.data_as(ctypes.c_void_p), ctypes.byref(st))
        t_adj = time.perf_counter() - t0
        if rc != 0:
            raise RuntimeError(s.lib.dgh_integrator_error(it.h).decode())
        g_ad = phis @ grad

        def objective(u):
            val = ctypes.c_double()
            rc2 = s.lib.dgh_dirk3_replay(it.h, np.ascontiguousarray(u).ctypes.data_as(ctypes.c_void_p),
                                         ctypes.byref(val))
            if rc2 != 0:
                raise RuntimeError(s.lib.dgh_integrator_error(it.h).decode())
            return val.value

        replay = objective(u0)
        t0 = time.perf_counter()
        g_fd = np.array([(objective(u0 + h * phi) - objective(u0 - h * phi)) / (2 * h) for phi in phis])
        t_fd = time.perf_counter() - t0
        rel = np.abs(g_ad - g_fd) / np.max(np.abs(g_ad))
        return {
            "config": f"{nx}x{nx} k={k} DIRK3 CFL {cfl} steps {steps} checkpoints every {every}",
            "objective": st.objective, "objective_replayed": replay, "final_time": st.final_time,
            "forward_newton_updates": st.forward_newton, "adjoint_krylov": st.adjoint_krylov,
            "checkpoints": st.checkpoints, "recomputed_steps": st.recomputed_steps,
            "gradient_adjoint": g_ad.tolist(), "gradient_fd": g_fd.tolist(),
            "max_error_rel_to_max_gradient": float(rel.max()),
            "per_mode_rel_error": (np.abs(g_ad - g_fd) / np.abs(g_ad)).tolist(), "fd_step": h,
            "adjoint_seconds": t_adj, "fd_seconds_16_forward_runs": t_fd, "within_1e-6": bool(rel.max() <= 1e-6),
        }
    finally:
        it.close()
        s.close()


def main() -> None:
    p = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    p.add_argument("--nx", type=int, default=128)
    p.add_argument("--k", type=int, default=4)
    p.add_argument("--steps", type=int, default=20)
    p.add_argument("--every", type=int, default=5)
    p.add_argument("--cfl", type=float, default=2.0)
    p.add_argument("--h", type=float, default=1e-6)
    p.add_argument("--amplitude", type=float, default=0.02, help="scale of each mode (density units)")
    args = p.parse_args()
    print(json.dumps(gradient_check(args.nx, args.k, args.steps, args.every, args.cfl, args.h, args.amplitude)))


if __name__ == "__main__":
    main()
