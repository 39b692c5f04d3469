"""Pin the CPU oracle against the reference's own archived outputs (tests/golden/).

These tests validate the oracle itself: they run it (a C++ restatement of
YueWu2002/DG_HDG_Euler_Cpp) on the exact command lines the reference archived and compare
residual histories, Krylov counts, L2 errors and nodal solutions.
"""
import ctypes
import json
import os
import tempfile
from pathlib import Path

import numpy as np
import pytest

from conftest import GOLDEN, ROOT, assert_history_close, read_csv


def _flags_from_command(name):
    """Reference command line minus the executable, output prefix and the retired --alpha-deg."""
    argv = json.loads((GOLDEN / name).read_text())[1:]
    out, skip = [], False
    for i, a in enumerate(argv):
        if skip:
            skip = False
            continue
        if a in ("--prefix", "--alpha-deg"):
            skip = True
            continue
        out.append(a)
    return out


def test_gauss_rule_against_reference_fastgl(oracle_mod):
    """nodal_basis.hpp:12-23 uses Bogaert's fastgl; our Newton rule must agree to a few ulps."""
    ref = ROOT / "oracle" / "_ref" / "libfastgl_ref.so"
    if not ref.exists():
        pytest.skip("reference fastgl not compiled here (reference tree absent)")
    fl = ctypes.CDLL(str(ref))
    for n in list(range(1, 10)) + [20, 21, 23]:
        xr, wr = np.zeros(n), np.zeros(n)
        P = ctypes.POINTER(ctypes.c_double)
        fl.fastgl_rule(n, xr.ctypes.data_as(P), wr.ctypes.data_as(P))
        o = oracle_mod.Oracle(f"--nx 3 --ny 3 --k {min(n, 9) - 1}")
        if n <= 9:
            x, w = o.basis()
            ulp_x = np.abs(x - xr) / np.spacing(np.maximum(np.abs(xr), 1e-300))
            assert np.all((np.abs(x - xr) <= 4 * np.spacing(1.0))), (n, ulp_x)
            assert np.all(np.abs(w - wr) <= 4 * np.spacing(wr)), (n, w - wr)


@pytest.mark.parametrize("case", ["dirk3", "be", "entropy"])
def test_4x4_production_checks(oracle_mod, case):
    """code_test/2d/test_solver.py:13-21 on 4x4 k=2 with --method both --check-update."""
    flags = _flags_from_command(f"c4x4_{case}.command.json")
    with tempfile.TemporaryDirectory() as tmp:
        res = oracle_mod.run_cli(flags + ["--prefix", f"{tmp}/run"])
        assert res.returncode == 0, res.stderr
        ours_it = read_csv(f"{tmp}/run_iterations.csv")
        ours_sum = read_csv(f"{tmp}/run_summary.csv")
        ours_diff = read_csv(f"{tmp}/run_difference.csv")[0]
    ref_it = read_csv(GOLDEN / f"c4x4_{case}_iterations.csv")
    assert_history_close(ours_it, ref_it)
    ref_sum = read_csv(GOLDEN / f"c4x4_{case}_summary.csv")
    for a, b in zip(ours_sum, ref_sum):
        assert a["method"] == b["method"]
        assert a["newton_iterations"] == b["newton_iterations"]
        assert abs(int(a["krylov_iterations"]) - int(b["krylov_iterations"])) <= 2
        assert float(a["volume_dofs"]) == float(b["volume_dofs"])
        assert float(a["trace_dofs"]) == float(b["trace_dofs"])
        assert float(a["max_conservation_drift"]) <= 1e-10
        for key in ("final_time", "min_step", "max_step", "lx", "ly"):
            assert abs(float(a[key]) - float(b[key])) <= 1e-14 * abs(float(b[key])), key
    assert float(ours_diff["max_nodal"]) <= 1e-9


def test_first_dirk_nodal_solution(oracle_mod):
    """The only archived 2D nodal solution (4x4 k=2 DIRK3 CFL2 T0.02, DG and HDG)."""
    with tempfile.TemporaryDirectory() as tmp:
        res = oracle_mod.run_cli(["--nx", "4", "--ny", "4", "--k", "2", "--cfl", "2", "--T", "0.02",
                                  "--method", "both", "--ntol", "1e-12", "--ltol", "1e-12",
                                  "--prefix", f"{tmp}/run"])
        assert res.returncode == 0, res.stderr
        ours = read_csv(f"{tmp}/run_solution.csv")
        ours_sum = read_csv(f"{tmp}/run_summary.csv")
    ref = read_csv(GOLDEN / "first_dirk_solution.csv")
    assert len(ours) == len(ref) == 288
    keys = ["rho", "momentum_x", "momentum_y", "energy"]
    worst = 0.0
    for a, b in zip(ours, ref):
        assert (a["method"], a["cell"], a["node"]) == (b["method"], b["cell"], b["node"])
        for k in ("x", "y"):
            assert abs(float(a[k]) - float(b[k])) <= 1e-15
        for k in keys + [k + "_exact" for k in keys]:
            d = abs(float(a[k]) - float(b[k])) / max(abs(float(b[k])), 1e-300)
            worst = max(worst, d)
    assert worst <= 1e-10, worst
    ref_sum = read_csv(GOLDEN / "first_dirk_summary.csv")
    for a, b in zip(ours_sum, ref_sum):
        for k in ("rho_L2", "momentum_x_L2", "momentum_y_L2", "energy_L2"):
            assert abs(float(a[k]) - float(b[k])) <= 1e-10 * float(b[k]), k


@pytest.mark.slow
def test_64x64_k2_first_dirk3_step(oracle_mod):
    """Accuracy run n64 (config 64^2 k=2): the first DIRK3 step's 12 Newton updates per method."""
    flags = _flags_from_command("acc_n64.command.json")
    flags = [f for f in flags if f != "--no-save-solution"]
    i = flags.index("--T")
    flags = flags[:i] + flags[i + 2:] + ["--steps", "1", "--no-save-solution", "--threads", "8"]
    with tempfile.TemporaryDirectory() as tmp:
        res = oracle_mod.run_cli(flags + ["--prefix", f"{tmp}/run"])
        assert res.returncode == 0, res.stderr
        ours = read_csv(f"{tmp}/run_iterations.csv")
    ref = [r for r in read_csv(GOLDEN / "acc_n64_iterations.csv") if r["step"] == "0"]
    # --steps 1 does not truncate the step; the archived run's first step was not truncated either
    assert_history_close(ours, ref)


@pytest.mark.slow
@pytest.mark.parametrize("k", [2, pytest.param(8, marks=pytest.mark.skipif(
    not os.environ.get("DGH_SLOW_ORACLE"), reason="minutes of CPU; set DGH_SLOW_ORACLE=1 (the device test "
    "test_256_initial_residual_and_dt pins k = 8 against the same archived row)"))])
def test_256_first_update_residual_and_dt(oracle_mod, k):
    """Speed run 256^2 (BE CFL5): initial projected state, frozen speeds, dt and first rms."""
    ref = read_csv(GOLDEN / f"speed256_k{k}_dg_iterations.csv")[0]
    o = oracle_mod.Oracle(f"--nx 256 --ny 256 --k {k} --integrator be --steps 1 --cfl 5", threads=8)
    u = o.initial()
    dt = 5.0 / o.freeze(u)
    assert abs(dt - float(ref["dt"])) <= 1e-15 * dt
    o.set_stage(u, dt)
    rms = o.rms(o.residual(u))
    assert abs(rms - float(ref["residual_physical_rms"])) <= 1e-13 * rms


def test_accuracy_table_l2_errors_recorded():
    """The convergence table the GPU path is checked against (RESULTS.md:136-141)."""
    rows = {(r["method"], r["nx"]): r for r in read_csv(GOLDEN / "acc_convergence.csv")}
    assert abs(float(rows[("dg", "64")]["rho_L2"]) - 9.0130040970360289e-05) < 1e-18
    assert abs(float(rows[("dg", "256")]["rho_L2"]) - 1.738849266065954e-06) < 1e-18
