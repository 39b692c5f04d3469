"""FP32 HDG condensation (dgh_config.condense32) against the oracle's FP64 condensation and the
reference's archived runs.

The FP32 form factors every cell matrix in FP32 with FP32 accumulation, keeps the factors and
stores S in FP32, so its operators match the FP64 ones to FP32 accuracy: 2e-5 relative here
(FP32 LU of blocks up to 324 wide, conditioning ~1e2).  The Newton updates are refined in FP64
on the DG system to the reference's acceptance target, so whole updates and runs match the
FP64 results to 1e-10 (states) and the archived histories under the history rule of
tests/conftest.py, with rtol 1e-8 for Newton rows above the rounding floor: a row's residual
depends on the previous update's linear solve, which every form stops at ltol = 1e-12 relative to
the previous residual (~0.4), i.e. within ~4e-13 absolute; on rows near 1e-4 that is a few 1e-9
relative however the Krylov path differs.  The FP64 form, whose Krylov path is the reference's,
holds 1e-10.
"""
import ctypes
import subprocess
import tempfile

import numpy as np
import pytest

from conftest import GOLDEN, assert_history_close, read_csv

pytestmark = pytest.mark.gpu

F32_TOL = 2e-5


def direction(n, a=.31, b=.79):
    i = np.arange(n)
    return .2 * np.sin(a * i) + .1 * np.cos(b * i)


def rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def np_(t):
    return t.detach().cpu().numpy()


@pytest.mark.parametrize("nx,ny,k", [(4, 4, 2), (3, 4, 4), (3, 3, 8), (5, 3, 1), (4, 3, 3)])
def test_condense32_operators_against_oracle(oracle_mod, nx, ny, k):
    from dg_hdg_euler_cpp_b200.solver import Solver

    o = oracle_mod.Oracle(f"--nx {nx} --ny {ny} --k {k} --cfl 2 --integrator be --steps 1")
    s = Solver(nx=nx, ny=ny, k=k, cfl=2.0, integrator="be", steps=1, method="hdg", precision="mixed", condense32=1)
    uo = o.initial()
    o.freeze(uo)
    s.freeze(s.tensor(uo))
    o.set_stage(uo, .003)
    s.set_stage(s.tensor(uo), .003)
    up = uo + 1e-3 * direction(uo.size)
    r = o.residual(up)
    o.hdg_refresh(up, r)
    s.hdg_refresh_projected(s.tensor(up), s.tensor(r))
    assert rel(np_(s.hdg_rhs()), o.hdg_rhs()) <= F32_TOL
    dl = direction(o.trace_size)
    assert rel(np_(s.hdg_apply(s.tensor(dl))), o.hdg_apply(dl)) <= F32_TOL
    for face in sorted({0, o.cells - 1, o.cells, o.faces - 1}):
        assert rel(s.hdg_block(face, face), o.hdg_block(face, face)) <= F32_TOL
    assert rel(np_(s.hdg_recover(s.tensor(dl))), o.hdg_recover(dl)) <= F32_TOL
    assert rel(np_(s.hdg_recovered_residual(s.tensor(dl))), o.hdg_recovered_residual(dl)) <= 1e-12
    # retarget to another volume residual: the oracle re-condenses with it (same state)
    r2 = o.residual(up + 1e-3 * direction(uo.size, .17, .53))
    s.hdg_retarget(s.tensor(r2))
    o.hdg_refresh(up, r2)
    assert rel(np_(s.hdg_rhs()), o.hdg_rhs()) <= F32_TOL
    assert rel(np_(s.hdg_recover(s.tensor(dl))), o.hdg_recover(dl)) <= F32_TOL
    # the kept factors solve the cell systems: recover(0) = -y = -A^{-1} r2
    y = -np_(s.hdg_recover(s.tensor(np.zeros(o.trace_size))))
    assert rel(y, -o.hdg_recover(np.zeros(o.trace_size))) <= F32_TOL
    s.close()


def test_condense32_fp64_context_refuses_retarget(oracle_mod):
    from dg_hdg_euler_cpp_b200.solver import DGHError, Solver

    o = oracle_mod.Oracle("--nx 3 --ny 3 --k 2 --cfl 2 --integrator be --steps 1")
    s = Solver(nx=3, ny=3, k=2, cfl=2.0, integrator="be", steps=1, method="hdg")
    u = s.tensor(o.initial())
    s.freeze(u)
    s.set_stage(u, .003)
    s.hdg_refresh_projected(u, s.residual(u))
    with pytest.raises(DGHError, match="condense32"):
        s.hdg_retarget(s.residual(u))
    s.close()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_condense32_newton_update_matches_oracle(oracle_mod, precision):
    """One backward-Euler Newton update at 8 x 8, k = 3 with the FP32 condensation and FP64
    refinement against the oracle's FP64 DG update: state within 1e-10 of the largest value."""
    from dg_hdg_euler_cpp_b200.solver import Integrator, Solver

    nx, ny, k, cfl = 8, 8, 3, 1.0
    o = oracle_mod.Oracle(f"--nx {nx} --ny {ny} --k {k} --cfl {cfl} --integrator be --steps 1 --restart 20")
    u0 = o.initial()
    dt = cfl / o.freeze(u0)
    o.set_stage(u0, dt)
    r0 = o.residual(u0)
    o.dg_refresh(u0)
    o.dg_precond_refresh()
    du, _, _, _ = o.gmres(0, -r0, 20, 1500, 1e-12)
    s = Solver(nx=nx, ny=ny, k=k, cfl=cfl, integrator="be", steps=1, newton_steps=1, restart=20, method="hdg",
               precision=precision, condense32=1)
    it = Integrator(s, "hdg")
    it.stage_begin(s.tensor(u0))
    row = it.update()
    assert row["dg_linear_relative_residual"] <= 1e-11
    state = s.vec()
    s.lib.dgh_axpby(s.h, 1.0, ctypes.c_void_p(it.state_ptr()), 0.0, ctypes.c_void_p(it.state_ptr()),
                    ctypes.c_void_p(state.data_ptr()), state.numel())
    s.lib.dgh_sync(s.h)
    err = np.max(np.abs(np_(state) - (u0 + row["damping"] * du))) / np.max(np.abs(u0))
    assert err <= 1e-10, err
    it.close()
    s.close()


def run_cli(args):
    from dg_hdg_euler_cpp_b200 import BIN_PATH

    return subprocess.run([str(BIN_PATH), *args], capture_output=True, text=True, timeout=900)


@pytest.mark.parametrize("case,extra", [("dirk3", []), ("be", ["--integrator", "be"])])
def test_condense32_cli_4x4_histories(case, extra):
    """The 4x4 production checks (code_test/2d/test_solver.py:13-21) with the FP32 condensation:
    the archived histories (1e-10 above the rounding floor), Newton counts and L2 errors."""
    with tempfile.TemporaryDirectory() as tmp:
        res = run_cli(["--nx", "4", "--ny", "4", "--k", "2", "--cfl", "2", "--method", "both", "--ntol", "1e-12",
                       "--ltol", "1e-12", "--no-save-solution", "--T", "0.02", "--condensation", "fp32",
                       "--precision", "mixed", *extra, "--prefix", f"{tmp}/run"])
        assert res.returncode == 0, res.stderr + res.stdout
        ours = read_csv(f"{tmp}/run_iterations.csv")
        summ = read_csv(f"{tmp}/run_summary.csv")
    ref = read_csv(GOLDEN / f"c4x4_{case}_iterations.csv")
    # Krylov counts of the refined form are the sum over its passes: not compared
    assert_history_close(ours, ref, rtol=1e-8, krylov_slack=10 ** 6)
    for a, b in zip(summ, read_csv(GOLDEN / f"c4x4_{case}_summary.csv")):
        assert a["newton_iterations"] == b["newton_iterations"]
        for key in ("rho_L2", "momentum_x_L2", "momentum_y_L2", "energy_L2"):
            assert abs(float(a[key]) - float(b[key])) <= 1e-10 * float(b[key]), key


def test_condense32_cli_64x64_k2_accuracy_run():
    """The 64^2 Q2 DIRK3 accuracy run to T = 0.2 with the FP32 condensation: the HDG history
    against the archived one, equal Newton counts and the L2 errors to 1e-9."""
    import json

    argv = json.loads((GOLDEN / "acc_n64.command.json").read_text())[1:]
    flags, i = [], 0
    while i < len(argv):
        if argv[i] in ("--alpha-deg", "--prefix"):
            i += 2
            continue
        flags.append(argv[i])
        i += 1
    flags[flags.index("--method") + 1] = "hdg"
    with tempfile.TemporaryDirectory() as tmp:
        res = run_cli([*flags, "--condensation", "fp32", "--precision", "mixed", "--graph", "--prefix", f"{tmp}/r"])
        assert res.returncode == 0, res.stderr + res.stdout
        ours = read_csv(f"{tmp}/r_iterations.csv")
        summ = read_csv(f"{tmp}/r_summary.csv")[0]
    ref = [r for r in read_csv(GOLDEN / "acc_n64_iterations.csv") if r["method"] == "hdg"]
    assert_history_close(ours, ref, rtol=1e-8, krylov_slack=10 ** 6)
    conv = {(r["method"], r["nx"]): r for r in read_csv(GOLDEN / "acc_convergence.csv")}[("hdg", "64")]
    assert summ["newton_iterations"] == conv["newton_iterations"]
    for key in ("rho_L2", "momentum_x_L2", "momentum_y_L2", "energy_L2"):
        assert abs(float(summ[key]) - float(conv[key])) <= 1e-9 * float(conv[key]), key


def test_forcing_floor_cli_64x64_k2_accuracy_run():
    """The 64^2 Q2 DIRK3 accuracy run with the forcing floor (linear solves stop at the absolute
    level no later test sees) and the FP32 forms: Newton counts equal to the archived run's, the
    Newton rows on the history rule down to the 1e-10 r0 floor, the L2 errors to 1e-9."""
    import json

    argv = json.loads((GOLDEN / "acc_n64.command.json").read_text())[1:]
    flags, i = [], 0
    while i < len(argv):
        if argv[i] in ("--alpha-deg", "--prefix"):
            i += 2
            continue
        flags.append(argv[i])
        i += 1
    with tempfile.TemporaryDirectory() as tmp:
        res = run_cli([*flags, "--condensation", "fp32", "--precision", "mixed16", "--forcing", "1", "--graph",
                       "--prefix", f"{tmp}/r"])
        assert res.returncode == 0, res.stderr + res.stdout
        ours = read_csv(f"{tmp}/r_iterations.csv")
        summ = {r["method"]: r for r in read_csv(f"{tmp}/r_summary.csv")}
    ref = read_csv(GOLDEN / "acc_n64_iterations.csv")
    conv = {(r["method"], r["nx"]): r for r in read_csv(GOLDEN / "acc_convergence.csv")}
    for method in ("dg", "hdg"):
        assert_history_close([r for r in ours if r["method"] == method], [r for r in ref if r["method"] == method],
                             rtol=1e-8, krylov_slack=10 ** 6)
        c = conv[(method, "64")]
        assert summ[method]["newton_iterations"] == c["newton_iterations"]
        assert int(summ[method]["krylov_iterations"]) < int(c["krylov_iterations"])
        for key in ("rho_L2", "momentum_x_L2", "momentum_y_L2", "energy_L2"):
            assert abs(float(summ[method][key]) - float(c[key])) <= 1e-9 * float(c[key]), key
