"""FP16 storage of the DG block-Jacobi factors (DGH_PRECISION_MIXED16, an extra form below the
FP32 factors): the factors are computed in FP64, every row of U is divided by its largest entry
(the FP32 row scale is kept), and both sweeps run in FP32.

Tolerances: the preconditioner solve matches the oracle's FP64 block Jacobi to 5e-3 relative
(FP16 keeps 11 significant bits; the triangular sweeps of up to 324 rows amplify that by the
blocks' conditioning, ~1e2 at these steps); GMRES on the FP64 operator still reaches the same
1e-12 tolerance, so its solution agrees with the oracle's to 1e-9 and whole runs match the
archived histories under the history rule of tests/conftest.py with rtol 1e-8 above the rounding
floor (a row's residual depends on the previous update's linear solve, stopped at ltol = 1e-12
relative to the previous residual: a few 1e-9 relative on rows near 1e-4 for any Krylov path
other than the reference's).
"""
import subprocess
import tempfile

import numpy as np
import pytest

from conftest import GOLDEN, assert_history_close, read_csv

pytestmark = pytest.mark.gpu

CASES = [(4, 4, 2), (5, 3, 1), (3, 4, 4), (3, 3, 8), (6, 5, 0), (4, 3, 3)]


def direction(n):
    i = np.arange(n)
    return .2 * np.sin(.31 * i) + .1 * np.cos(.79 * i)


def rel(a, b):
    return float(np.max(np.abs(np.asarray(a) - np.asarray(b))) / np.max(np.abs(b)))


def pair(oracle_mod, nx, ny, k):
    from dg_hdg_euler_cpp_b200.solver import Solver

    o = oracle_mod.Oracle(f"--nx {nx} --ny {ny} --k {k} --cfl 2 --integrator be --steps 1")
    s = Solver(nx=nx, ny=ny, k=k, cfl=2.0, integrator="be", steps=1, method="dg", precision="mixed16")
    uo = o.initial()
    ug = s.tensor(uo)
    o.freeze(uo)
    s.freeze(ug)
    o.set_stage(uo, .003)
    s.set_stage(ug, .003)
    up = uo + 1e-3 * direction(uo.size)
    o.dg_refresh(up)
    s.dg_refresh(s.tensor(up))
    o.dg_precond_refresh()
    s.precond_refresh("dg")
    return o, s, up


@pytest.mark.parametrize("nx,ny,k", CASES)
def test_half_factor_precond_against_oracle(oracle_mod, nx, ny, k):
    o, s, _ = pair(oracle_mod, nx, ny, k)
    d = direction(o.size)
    zg = s.precond_apply("dg", s.tensor(d)).cpu().numpy()
    assert rel(zg, o.dg_precond_apply(d)) <= 5e-3
    s.close()


@pytest.mark.parametrize("nx,ny,k", [(4, 4, 2), (3, 3, 8)])
def test_half_factor_gmres_reaches_fp64_solution(oracle_mod, nx, ny, k):
    from dg_hdg_euler_cpp_b200.solver import DGHError

    o, s, up = pair(oracle_mod, nx, ny, k)
    r = o.residual(up)
    xo, ito, _, _ = o.gmres(0, -r, 20, 1500, 1e-12)
    xg, itg, relg, _ = s.gmres("dg", s.tensor(-r), 1500, 1e-12)
    assert relg <= 1e-12 and itg >= ito
    assert rel(xg.cpu().numpy(), xo) <= 1e-9
    with pytest.raises(DGHError, match="FP64 or FP32 factors"):
        s.precond_apply("dg_t", s.tensor(r))
    s.close()


@pytest.mark.parametrize("case,extra", [("dirk3", []), ("be", ["--integrator", "be"])])
def test_half_factor_cli_4x4_histories(case, extra):
    from dg_hdg_euler_cpp_b200 import BIN_PATH

    with tempfile.TemporaryDirectory() as tmp:
        res = subprocess.run([str(BIN_PATH), "--nx", "4", "--ny", "4", "--k", "2", "--cfl", "2", "--method", "dg",
                              "--ntol", "1e-12", "--ltol", "1e-12", "--no-save-solution", "--T", "0.02",
                              "--precision", "mixed16", *extra, "--prefix", f"{tmp}/run"], capture_output=True,
                             text=True, timeout=600)
        assert res.returncode == 0, res.stderr + res.stdout
        ours = read_csv(f"{tmp}/run_iterations.csv")
        summ = read_csv(f"{tmp}/run_summary.csv")[0]
    ref = [r for r in read_csv(GOLDEN / f"c4x4_{case}_iterations.csv") if r["method"] == "dg"]
    assert_history_close(ours, ref, rtol=1e-8, krylov_slack=10 ** 6)  # FP16 factors change the Krylov counts
    refs = [r for r in read_csv(GOLDEN / f"c4x4_{case}_summary.csv") if r["method"] == "dg"][0]
    assert summ["newton_iterations"] == refs["newton_iterations"]
    for key in ("rho_L2", "momentum_x_L2", "momentum_y_L2", "energy_L2"):
        assert abs(float(summ[key]) - float(refs[key])) <= 1e-10 * float(refs[key]), key
