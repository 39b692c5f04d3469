"""The 1D device path (dgh_config.dim = 1) against the 1D CPU oracle and the reference's
archived 1D runs.

Tolerances: residual, J*v, blocks, traces and norms 1e-12 relative (summation order only);
block solves 1e-10 (FP64 LU) or 1e-4 (FP32 factors); GMRES solutions 1e-9 (both solve to
1e-12).  Archived runs: the comparisons of tests/conftest.py, with --restart 20 (the archived
1D runs used GMRES(20); see tests/test_oracle1d_golden.py).
"""
import subprocess
import tempfile

import numpy as np
import pytest

from conftest import GOLDEN, assert_history_close, read_csv

pytestmark = pytest.mark.gpu

CASES = [(5, 0, 0), (6, 1, 0), (7, 2, 0), (5, 3, 0), (4, 8, 0), (5, 1, 4), (6, 3, 6), (3, 8, 12)]


def direction(n, a=.7, b=1.9):
    i = np.arange(n)
    return np.sin(a * i) + .2 * np.cos(b * i)


def rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def np_(t):
    return t.detach().cpu().numpy()


def setup(oracle_mod, cells, k, quad, precision="fp64", step=.003):
    from dg_hdg_euler_cpp_b200.solver import Solver

    o = oracle_mod.Oracle1D(f"--cells {cells} --k {k} --quad {quad} --integrator be --steps 1")
    s = Solver(dim=1, cells=cells, k=k, quad=quad, cfl=2.0, integrator="be", steps=1, method="both",
               precision=precision)
    u = o.initial()
    ug = s.tensor(u)
    o.freeze(u)
    s.freeze(ug)
    o.set_stage(u, step)
    s.set_stage(ug, step)
    return o, s, u


@pytest.mark.parametrize("cells,k,quad", CASES)
def test_problem_kernels(oracle_mod, cells, k, quad):
    from dg_hdg_euler_cpp_b200.solver import Solver

    o = oracle_mod.Oracle1D(f"--cells {cells} --k {k} --quad {quad}")
    s = Solver(dim=1, cells=cells, k=k, quad=quad, method="both")
    assert (s.size, s.trace_size, s.block, s.cells) == (o.size, o.trace_size, o.block, o.cells)
    uo = o.initial()
    assert rel(np_(s.initial()), uo) <= 1e-13
    ug = s.tensor(uo)
    rate_o, rate_g = o.freeze(uo), s.freeze(ug)
    assert abs(rate_o - rate_g) <= 1e-14 * rate_o
    assert rel(s.speeds(), o.speeds()) <= 1e-14
    o.set_stage(uo, .003)
    s.set_stage(ug, .003)
    up = uo + 1e-3 * direction(uo.size)
    assert rel(np_(s.residual(s.tensor(up))), o.residual(up)) <= 1e-12
    r = o.residual(up)
    assert abs(s.dual_norm(s.tensor(r)) - o.dual_norm(r)) <= 1e-13 * o.dual_norm(r)
    assert abs(s.residual_rms(s.tensor(r)) - o.rms(r)) <= 1e-13 * o.rms(r)
    assert s.admissible(s.tensor(up)) and o.admissible(up)
    for idx, val in ((0, -1.0), (4, np.nan)):
        bad = up.copy()
        bad[idx] = val
        assert s.admissible(s.tensor(bad)) is False and o.admissible(bad) is False
    assert rel(np_(s.trace(s.tensor(up))), o.trace(up)) <= 1e-13
    assert rel(s.integral(s.tensor(up)), o.integral(up)) <= 1e-13
    assert rel(s.l2_error(s.tensor(up), .05), o.l2_error(up, .05)) <= 1e-11


@pytest.mark.parametrize("cells,k,quad", CASES)
def test_dg_operator_blocks_and_precond(oracle_mod, cells, k, quad):
    o, s, u = setup(oracle_mod, cells, k, quad)
    up = u + 1e-4 * direction(u.size)
    o.dg_refresh(up)
    s.dg_refresh(s.tensor(up))
    d = direction(u.size, .31, .79)
    assert rel(np_(s.dg_apply(s.tensor(d))), o.dg_apply(d)) <= 1e-12
    for cell in sorted({0, cells // 2, cells - 1}):
        assert rel(s.dg_block(cell, cell), o.dg_block(cell, cell)) <= 1e-13
    o.dg_precond_refresh()
    s.precond_refresh("dg")
    assert rel(np_(s.precond_apply("dg", s.tensor(d))), o.dg_precond_apply(d)) <= 1e-10
    # the transposed solve: A^T z = d per block
    zt = np_(s.precond_apply("dg_t", s.tensor(d)))
    m = o.block
    for cell in range(cells):
        a = o.dg_block(cell, cell)
        ref = np.linalg.solve(a.T, d[cell * m:(cell + 1) * m])
        assert np.max(np.abs(zt[cell * m:(cell + 1) * m] - ref)) <= 1e-10 * np.max(np.abs(ref))


@pytest.mark.parametrize("cells,k,quad", CASES)
def test_hdg_condensation(oracle_mod, cells, k, quad):
    o, s, u = setup(oracle_mod, cells, k, quad)
    up = u + 1e-3 * direction(u.size)
    r = o.residual(up)
    o.hdg_refresh(up, r)
    s.hdg_refresh_projected(s.tensor(up), s.tensor(r))
    assert rel(np_(s.hdg_rhs()), o.hdg_rhs()) <= 1e-11
    dl = direction(o.trace_size, .31, .79)
    assert rel(np_(s.hdg_apply(s.tensor(dl))), o.hdg_apply(dl)) <= 1e-11
    for f in sorted({0, cells // 2, cells - 1}):
        assert rel(s.hdg_block(f, f), o.hdg_block(f, f)) <= 1e-11
    assert rel(np_(s.hdg_recover(s.tensor(dl))), o.hdg_recover(dl)) <= 1e-11
    # the device takes the Schur error e = S dl - rhs; the oracle forms it from dl
    e = o.hdg_apply(dl) - o.hdg_rhs()
    assert rel(np_(s.hdg_recovered_residual(s.tensor(e))), o.hdg_recovered_residual(dl)) <= 1e-11
    o.hdg_precond_refresh()
    s.precond_refresh("hdg")
    assert rel(np_(s.precond_apply("hdg", s.tensor(dl))), o.hdg_precond_apply(dl)) <= 1e-10


@pytest.mark.parametrize("cells,k,quad", [(8, 2, 0), (6, 3, 5), (5, 8, 0)])
def test_gmres_dg_and_hdg(oracle_mod, cells, k, quad):
    o, s, u = setup(oracle_mod, cells, k, quad, step=.05)
    up = u + 1e-3 * direction(u.size)
    r = o.residual(up)
    o.dg_refresh(up)
    s.dg_refresh(s.tensor(up))
    o.dg_precond_refresh()
    s.precond_refresh("dg")
    xo, ito, _, _ = o.gmres(0, -r, 20, 1500, 1e-12)
    xg, itg, relg, resg = s.gmres("dg", s.tensor(-r), 1500, 1e-12)
    assert abs(ito - itg) <= 1 and relg <= 1e-12
    assert rel(np_(xg), xo) <= 1e-9
    assert np.max(np.abs(np_(resg) - (-r - o.dg_apply(np_(xg))))) <= 1e-11 * np.max(np.abs(r))
    o.hdg_refresh(up, r)
    s.hdg_refresh_projected(s.tensor(up), s.tensor(r))
    o.hdg_precond_refresh()
    s.precond_refresh("hdg")
    rhs = o.hdg_rhs()
    lo, ito, _, _ = o.gmres(1, rhs, 20, 1500, 1e-12)
    lg, itg, _, _ = s.gmres("hdg", s.tensor(rhs), 1500, 1e-12)
    assert abs(ito - itg) <= 1
    assert rel(np_(lg), lo) <= 1e-9


@pytest.mark.parametrize("cells,k,quad", [(5, 2, 0), (4, 3, 6)])
def test_mixed_precision_precond(oracle_mod, cells, k, quad):
    o, s, u = setup(oracle_mod, cells, k, quad, precision="mixed")
    o.dg_refresh(u)
    s.dg_refresh(s.tensor(u))
    o.dg_precond_refresh()
    s.precond_refresh("dg")
    d = direction(u.size)
    assert rel(np_(s.precond_apply("dg", s.tensor(d))), o.dg_precond_apply(d)) <= 1e-4


def run_cli(args):
    from dg_hdg_euler_cpp_b200 import BIN1D_PATH

    return subprocess.run([str(BIN1D_PATH), *args], capture_output=True, text=True, timeout=900)


@pytest.mark.parametrize("case,args,krylov,rtol", [
    ("be_update", ["--cells", "32", "--k", "3", "--integrator", "be", "--steps", "1", "--check-update"], 1, 1e-10),
    ("dirk_smoke", ["--cells", "16", "--k", "2", "--integrator", "ssp-dirk3", "--T", "0.02", "--check-update"], 1,
     1e-10),
    ("k8_n32", ["--cells", "32", "--k", "8", "--integrator", "be", "--steps", "1"], 2, 1e-8),
])
def test_cli_archived_1d_runs(case, args, krylov, rtol):
    """code_test/1d/test_solver.py:16-21 through the device CLI, against the archived runs."""
    with tempfile.TemporaryDirectory() as tmp:
        res = run_cli([*args, "--method", "both", "--cfl", "2", "--precond", "block-jacobi", "--ntol", "1e-12",
                       "--ltol", "1e-12", "--restart", "20", "--prefix", f"{tmp}/run"])
        assert res.returncode == 0, res.stderr + res.stdout
        its = read_csv(f"{tmp}/run_iterations.csv")
        summ = read_csv(f"{tmp}/run_summary.csv")
        sol = read_csv(f"{tmp}/run_solution.csv")
        diff = read_csv(f"{tmp}/run_difference.csv")[0]
    assert_history_close(its, read_csv(GOLDEN / f"d1_{case}_iterations.csv"), rtol=rtol, krylov_slack=krylov)
    for a, b in zip(summ, read_csv(GOLDEN / f"d1_{case}_summary.csv")):
        for key in ("method", "cells", "k", "quad", "steps", "newton_iterations", "volume_dofs", "trace_dofs"):
            assert a[key] == b[key], key
        assert float(a["max_conservation_drift"]) <= 1e-10
        for key in ("rho_L2", "momentum_L2", "energy_L2"):
            assert abs(float(a[key]) - float(b[key])) <= 1e-11 * float(b[key]), key
    ref = read_csv(GOLDEN / f"d1_{case}_solution.csv")
    assert len(sol) == len(ref)
    worst = max(abs(float(a[k]) - float(b[k])) / abs(float(b[k])) for a, b in zip(sol, ref)
                for k in ("rho", "momentum", "energy"))
    assert worst <= 1e-12, worst
    assert float(diff["max_nodal"]) <= 1e-9


def test_cli_accuracy_configuration_n64_k2():
    """The 1D accuracy configuration (64 cells, k=2, DIRK3 CFL 2, T=0.2): Newton count and L2
    errors against accuracy_test/results/1d_intel_20261019/convergence_intel_20261019.csv."""
    ref = [r for r in read_csv(GOLDEN / "d1_convergence.csv") if r["cells"] == "64"]
    with tempfile.TemporaryDirectory() as tmp:
        res = run_cli(["--cells", "64", "--k", "2", "--integrator", "ssp-dirk3", "--T", "0.2", "--method", "both",
                       "--cfl", "2", "--ntol", "1e-12", "--ltol", "1e-12", "--restart", "20", "--prefix", f"{tmp}/run"])
        assert res.returncode == 0, res.stderr
        summ = read_csv(f"{tmp}/run_summary.csv")
    for a in summ:
        b = next(r for r in ref if r["method"] == a["method"])
        assert (a["volume_dofs"], a["trace_dofs"]) == ("576", "192")
        assert a["newton_iterations"] == b["newton_iterations"] and a["steps"] == b["steps"]
        assert abs(int(a["krylov_iterations"]) - int(b["krylov_iterations"])) <= 4
        for key in ("rho_L2", "momentum_L2", "energy_L2"):
            assert abs(float(a[key]) - float(b[key])) <= 1e-9 * float(b[key]), key


@pytest.mark.parametrize("k,quad,integrator", [(3, 6, "ssp-dirk3"), (2, 0, "be"), (5, 9, "be")])
def test_advance_matches_oracle_with_overintegration(oracle_mod, k, quad, integrator):
    """TimeIntegrator::advance on 10 cells, both methods, the device against the oracle
    (over-integrated rules have no archived run)."""
    from dg_hdg_euler_cpp_b200.solver import Solver

    args = f"--cells 10 --k {k} --quad {quad} --cfl 1 --integrator {integrator} --T 0.05 --restart 20"
    o = oracle_mod.Oracle1D(args)
    u0 = o.initial()
    for method in ("dg", "hdg"):
        so, st_o, _ = o.advance(method, u0)
        s = Solver(dim=1, cells=10, k=k, quad=quad, cfl=1.0, integrator=integrator, final_time=0.05, restart=20,
                   method=method)
        sg, st_g, _ = s.advance(method, u0)
        assert np.max(np.abs(sg - so)) <= 1e-10 * np.max(np.abs(so))
        assert st_g["newton_iterations"] == st_o["newton_iterations"]
        assert abs(st_g["krylov_iterations"] - st_o["krylov_iterations"]) <= 2 * st_o["newton_iterations"]
        assert st_g["conservation_drift"] <= 1e-12
        s.close()


def test_mixed_precision_run_matches_fp64():
    """The FP32 block-Jacobi factors change only the Krylov path: the 1D BE run's state agrees
    with the FP64 run to the linear tolerance."""
    from dg_hdg_euler_cpp_b200.solver import Solver

    out = {}
    for precision in ("fp64", "mixed"):
        s = Solver(dim=1, cells=32, k=3, cfl=2.0, integrator="be", steps=1, restart=20, method="dg",
                   precision=precision)
        u0 = s.initial().cpu().numpy()
        out[precision] = s.advance("dg", u0)
        s.close()
    (a, sa, _), (b, sb, _) = out["fp64"], out["mixed"]
    assert sa["newton_iterations"] == sb["newton_iterations"]
    assert np.max(np.abs(a - b)) <= 1e-10 * np.max(np.abs(a))


def test_device_errors_use_the_reference_messages():
    from dg_hdg_euler_cpp_b200.solver import DGHError, Solver

    s = Solver(dim=1, cells=4, k=2, method="dg")
    u = s.initial()
    with pytest.raises(DGHError, match="Freeze the wave speeds"):
        s.residual(u)
    s.freeze(u)
    s.set_stage(u, .01)
    s.dg_refresh(u)
    with pytest.raises(DGHError, match="built for the 2D operator only"):
        s.dg_apply_T(u)
    bad = u.clone()
    bad[0] = -5.0  # density at the node nearest x = -1: the left trace of cell 0 turns negative
    with pytest.raises(DGHError, match="Invalid frozen face state"):
        s.freeze(bad)


# ---- block ILU(0) (--precond block-ilu0, block_ilu.cpp:15-84, natural ordering) ---------------
@pytest.mark.parametrize("cells,k,quad,precision,tol", [(8, 2, 0, "fp64", 1e-10), (6, 3, 6, "fp64", 1e-10),
                                                        (5, 8, 0, "fp64", 1e-10), (3, 1, 0, "fp64", 1e-10),
                                                        (7, 3, 0, "mixed", 1e-4)])
def test_block_ilu0_precond(oracle_mod, cells, k, quad, precision, tol):
    """The ILU(0) factors of the periodic DG and trace block patterns and their two sweeps
    against the oracle's restatement (FP64: 1e-10; FP32 factors: 1e-4)."""
    from dg_hdg_euler_cpp_b200.solver import Solver

    o = oracle_mod.Oracle1D(f"--cells {cells} --k {k} --quad {quad} --integrator be --steps 1 --precond block-ilu0")
    s = Solver(dim=1, cells=cells, k=k, quad=quad, cfl=2.0, integrator="be", steps=1, method="both",
               precision=precision, precond="block-ilu0")
    u = o.initial()
    ug = s.tensor(u)
    o.freeze(u)
    s.freeze(ug)
    o.set_stage(u, .05)
    s.set_stage(ug, .05)
    up = u + 1e-3 * direction(u.size)
    o.dg_refresh(up)
    s.dg_refresh(s.tensor(up))
    o.dg_precond_refresh()
    s.precond_refresh("dg")
    d = direction(u.size, .31, .79)
    assert rel(np_(s.precond_apply("dg", s.tensor(d))), o.dg_precond_apply(d)) <= tol
    r = o.residual(up)
    o.hdg_refresh(up, r)
    s.hdg_refresh_projected(s.tensor(up), s.tensor(r))
    o.hdg_precond_refresh()
    s.precond_refresh("hdg")
    dl = direction(o.trace_size, .31, .79)
    assert rel(np_(s.precond_apply("hdg", s.tensor(dl))), o.hdg_precond_apply(dl)) <= tol
    s.close()


@pytest.mark.parametrize("k,integrator", [(2, "ssp-dirk3"), (4, "be")])
def test_block_ilu0_advance_matches_oracle(oracle_mod, k, integrator):
    """TimeIntegrator::advance with block ILU(0) on 12 cells, both methods, device vs oracle."""
    from dg_hdg_euler_cpp_b200.solver import Solver

    args = f"--cells 12 --k {k} --cfl 2 --integrator {integrator} --T 0.05 --restart 20 --precond block-ilu0"
    o = oracle_mod.Oracle1D(args)
    u0 = o.initial()
    for method in ("dg", "hdg"):
        so, st_o, _ = o.advance(method, u0)
        s = Solver(dim=1, cells=12, k=k, cfl=2.0, integrator=integrator, final_time=0.05, restart=20, method=method,
                   precond="block-ilu0")
        sg, st_g, _ = s.advance(method, u0)
        assert np.max(np.abs(sg - so)) <= 1e-10 * np.max(np.abs(so))
        assert st_g["newton_iterations"] == st_o["newton_iterations"]
        assert abs(st_g["krylov_iterations"] - st_o["krylov_iterations"]) <= st_o["newton_iterations"]
        s.close()


def test_block_ilu0_cli_matches_oracle_cli(oracle_mod):
    """dgh1d --precond block-ilu0 against the oracle's CLI on the same run: histories, Krylov
    counts and L2 errors."""
    args = ["--cells", "32", "--k", "3", "--steps", "2", "--method", "both", "--cfl", "2", "--restart", "20",
            "--precond", "block-ilu0"]
    with tempfile.TemporaryDirectory() as tmp:
        res = run_cli([*args, "--prefix", f"{tmp}/gpu"])
        assert res.returncode == 0, res.stderr + res.stdout
        oracle_mod.run_cli_1d([*args, "--prefix", f"{tmp}/cpu"])
        its, ref = read_csv(f"{tmp}/gpu_iterations.csv"), read_csv(f"{tmp}/cpu_iterations.csv")
        summ, sref = read_csv(f"{tmp}/gpu_summary.csv"), read_csv(f"{tmp}/cpu_summary.csv")
    assert_history_close(its, ref, rtol=1e-10, krylov_slack=1)
    for a, b in zip(summ, sref):
        assert a["preconditioner"] == b["preconditioner"] == "block-ilu0"
        for key in ("rho_L2", "momentum_L2", "energy_L2"):
            assert abs(float(a[key]) - float(b[key])) <= 1e-10 * float(b[key]), key


def test_block_ilu0_nonfinite_block_message():
    """A non-finite block reaching the ILU(0) factorisation reports DenseLU's require() text
    (dense_lu.hpp:11-12) and stops the refresh."""
    from dg_hdg_euler_cpp_b200.solver import DGHError, Solver

    s = Solver(dim=1, cells=4, k=2, method="dg", precond="block-ilu0")
    u = s.initial()
    s.freeze(u)
    s.set_stage(u, .05)
    bad = u.clone()
    bad[3] = float("nan")
    s.dg_refresh(bad)  # the linearisation caches carry the NaN into the blocks
    with pytest.raises(DGHError, match="Nonfinite block LU input"):
        s.precond_refresh("dg")
    s.close()
