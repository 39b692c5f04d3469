"""Adjoint J^T w, the transposed block-Jacobi solve and the DIRK3 discrete adjoint.

Pins (no reference function exists for these; they are new): the transpose identity
<J^T w, v> = <w, J v> to 1e-12; J^T w against the transpose assembled from the oracle's coupling
blocks (DGOperator::block over the cartesian block graph, as check_2d.cpp:66-71 assembles J);
A^{-T} x against numpy solves with the oracle's blocks; and the gradient of the discrete adjoint
against central finite differences (h = 1e-6) of the same trajectory with dt and the frozen
speeds replayed, to 1e-6 relative.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def direction(n, a=.31, b=.79):
    i = np.arange(n)
    return .2 * np.sin(a * i) + .1 * np.cos(b * i)


def np_(t):
    return t.detach().cpu().numpy()


def setup(oracle_mod, nx, ny, k, precision="fp64"):
    from dg_hdg_euler_cpp_b200.solver import Solver

    o = oracle_mod.Oracle(f"--nx {nx} --ny {ny} --k {k} --cfl 2 --integrator be --steps 1")
    s = Solver(nx=nx, ny=ny, k=k, cfl=2.0, integrator="be", steps=1, method="dg", precision=precision)
    u = o.initial()
    o.freeze(u)
    ug = s.tensor(u)
    s.freeze(ug)
    o.set_stage(u, .004)
    s.set_stage(ug, .004)
    up = u + 1e-3 * direction(u.size)
    o.dg_refresh(up)
    s.dg_refresh(s.tensor(up))
    return o, s


@pytest.mark.parametrize("nx,ny,k", [(4, 4, 2), (3, 5, 1), (3, 3, 8), (8, 8, 4), (5, 4, 0)])
def test_adjoint_apply_identity_and_block_transpose(oracle_mod, nx, ny, k):
    o, s = setup(oracle_mod, nx, ny, k)
    v = direction(o.size)
    w = direction(o.size, .17, .53)
    jv = np_(s.dg_apply(s.tensor(v)))
    jtw = np_(s.dg_apply_T(s.tensor(w)))
    lhs, rhs = float(jtw @ v), float(w @ jv)
    assert abs(lhs - rhs) <= 1e-12 * max(abs(lhs), np.linalg.norm(jtw) * np.linalg.norm(v))
    ref = o.dg_apply_transpose(w)  # transpose of the five coupling blocks of every block row
    assert np.max(np.abs(jtw - ref)) <= 1e-12 * np.max(np.abs(ref))


@pytest.mark.parametrize("nx,ny,k,precision,tol", [(4, 4, 2, "fp64", 1e-10), (3, 3, 8, "fp64", 1e-10),
                                                   (3, 4, 4, "mixed", 1e-4)])
def test_transposed_block_solve(oracle_mod, nx, ny, k, precision, tol):
    o, s = setup(oracle_mod, nx, ny, k, precision)
    s.precond_refresh("dg")
    x = direction(o.size)
    z = np_(s.precond_apply("dg_t", s.tensor(x)))
    m = o.block
    for cell in range(o.cells):
        a = o.dg_block(cell, cell)
        ref = np.linalg.solve(a.T, x[cell * m:(cell + 1) * m])
        assert np.max(np.abs(z[cell * m:(cell + 1) * m] - ref)) <= tol * np.max(np.abs(ref))


def test_adjoint_gmres_solves_transposed_system(oracle_mod):
    o, s = setup(oracle_mod, 4, 4, 3)
    s.precond_refresh("dg")
    b = direction(o.size)
    psi, it, rel, res = s.gmres("dg_t", s.tensor(b), 1500, 1e-12)
    assert it > 0 and rel <= 1e-12
    r = b - np_(s.dg_apply_T(psi))
    w = 1.0 / o.mass
    assert np.sqrt(np.sum(r * r * w) / np.sum(b * b * w)) <= 1e-11


@pytest.mark.parametrize("integrator,steps,every", [("ssp-dirk3", 4, 2), ("be", 3, 2)])
def test_discrete_adjoint_gradient_matches_central_differences(integrator, steps, every):
    from dg_hdg_euler_cpp_b200 import _lib
    from dg_hdg_euler_cpp_b200.solver import Integrator, Solver

    nx, ny, k = 8, 8, 3  # a trajectory the reference algorithm itself keeps admissible
    s = Solver(nx=nx, ny=ny, k=k, cfl=0.3, integrator=integrator, steps=steps, method="dg", restart=20)
    it = Integrator(s, "dg")
    u0 = np_(s.initial())
    n = s.size
    plane = (k + 1) ** 2
    rho = ((np.arange(n) // plane) % 4) == 0
    grad = np.zeros(n)
    st = _lib.dgh_adjoint_stats()
    rc = s.lib.dgh_dirk3_adjoint(it.h, steps, every, u0.ctypes.data_as(ctypes.c_void_p),
                                 grad.ctypes.data_as(ctypes.c_void_p), ctypes.byref(st))
    assert rc == 0, s.lib.dgh_integrator_error(it.h).decode()
    assert st.recomputed_steps == steps and st.adjoint_krylov > 0

    def objective(u):
        val = ctypes.c_double()
        rc = s.lib.dgh_dirk3_replay(it.h, np.ascontiguousarray(u).ctypes.data_as(ctypes.c_void_p), ctypes.byref(val))
        assert rc == 0, s.lib.dgh_integrator_error(it.h).decode()
        return val.value

    assert abs(objective(u0) - st.objective) <= 1e-13 * st.objective
    h = 1e-6
    for seed in range(3):
        rng = np.random.default_rng(seed)
        phi = np.where(rho, rng.standard_normal(n), 0.0) * 0.05 * np.abs(u0)
        fd = (objective(u0 + h * phi) - objective(u0 - h * phi)) / (2 * h)
        ad = float(grad @ phi)
        assert abs(fd - ad) <= 1e-6 * abs(ad), (seed, fd, ad)
    it.close()
    s.close()


def dense_jacobian(o, nx: int, ny: int) -> np.ndarray:
    """J assembled from the oracle's DGOperator::block over the periodic cartesian block graph
    (each cell couples to itself and its four face neighbours), as check_2d.cpp:66-71 assembles
    the dense reference of `--linear direct` (direct.hpp:16-23)."""
    m = o.block
    J = np.zeros((o.size, o.size))
    for cell in range(o.cells):
        cx, cy = cell % nx, cell // nx
        for col in {cell, cy * nx + (cx + 1) % nx, cy * nx + (cx - 1) % nx, ((cy + 1) % ny) * nx + cx,
                    ((cy - 1) % ny) * nx + cx}:
            J[cell * m:(cell + 1) * m, col * m:(col + 1) * m] = o.dg_block(cell, col)
    return J


def test_adjoint_against_dense_jacobian_8x8_k4(oracle_mod):
    """8 x 8 cells at k = 4 (6,400 unknowns): the device's J^T w and its transposed GMRES solve
    (DGH_OP_DG_T with the transposed block-Jacobi preconditioner, ltol 1e-12) against the dense
    Jacobian assembled from the oracle's coupling blocks, its transpose product and a dense LU
    solve of J^T psi = b."""
    o, s = setup(oracle_mod, 8, 8, 4)
    J = dense_jacobian(o, 8, 8)
    v = direction(o.size)
    w = direction(o.size, .17, .53)
    # the dense J reproduces the matrix-free J v of both implementations
    assert np.max(np.abs(J @ v - o.dg_apply(v))) <= 1e-12 * np.max(np.abs(J @ v))
    jtw = np_(s.dg_apply_T(s.tensor(w)))
    ref = J.T @ w
    assert np.max(np.abs(jtw - ref)) <= 1e-12 * np.max(np.abs(ref))
    s.precond_refresh("dg")
    psi, it, rel, _ = s.gmres("dg_t", s.tensor(w), 1500, 1e-12)
    assert it > 0 and rel <= 1e-12
    dense = np.linalg.solve(J.T, w)
    err = np.max(np.abs(np_(psi) - dense)) / np.max(np.abs(dense))
    assert err <= 1e-9, err


def test_c5_discrete_adjoint_fourier_gradient_128_k4():
    """The discrete-adjoint configuration: 128^2 cells, k = 4, SSP-DIRK3 at CFL 2 for 20 steps,
    checkpoints every 5 steps, objective sum M rho^2 at the final time, gradient with respect to
    8 Fourier coefficients of the initial density perturbation.  Every coefficient of the
    adjoint gradient is within 1e-6 (relative to the largest) of central finite differences with
    h = 1e-6 of the replayed trajectory."""
    from dg_hdg_euler_cpp_b200.adjoint_check import gradient_check

    rec = gradient_check(nx=128, k=4, steps=20, every=5, cfl=2.0, h=1e-6)
    print("\n", rec)
    assert rec["recomputed_steps"] == 20 and rec["checkpoints"] >= 4
    assert abs(rec["objective_replayed"] - rec["objective"]) <= 1e-13 * rec["objective"]
    assert rec["max_error_rel_to_max_gradient"] <= 1e-6, rec
