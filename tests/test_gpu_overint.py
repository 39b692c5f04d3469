"""The 2D over-integrated volume rule (--quad Q > k+1) on the device against the oracle's
restatement (tests/test_oracle_overint.py pins the oracle): residual, CFL rate, admissibility at
the volume points, J*v, cell blocks, the block-Jacobi solve, the HDG condensation, whole runs
and the CLI, and the adjoint (J^T w, the transposed solve, the DIRK3 discrete-adjoint gradient).
Tolerances as in tests/test_gpu_parity.py and tests/test_gpu_adjoint.py."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CASES = [(4, 3, 2, 4), (3, 3, 3, 6), (3, 4, 1, 3)]


def direction(n, a=.7, b=1.9):
    i = np.arange(n)
    return np.sin(a * i) + .2 * np.cos(b * i)


def rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def np_(t):
    return t.detach().cpu().numpy()


def setup(oracle_mod, nx, ny, k, quad, precision="fp64"):
    from dg_hdg_euler_cpp_b200.solver import Solver

    o = oracle_mod.Oracle(f"--nx {nx} --ny {ny} --k {k} --quad {quad} --cfl 2 --integrator be --steps 1")
    s = Solver(nx=nx, ny=ny, k=k, quad=quad, cfl=2.0, integrator="be", steps=1, method="both", precision=precision)
    return o, s


@pytest.mark.parametrize("nx,ny,k,quad", CASES)
def test_residual_rate_jv_blocks_precond(oracle_mod, nx, ny, k, quad):
    o, s = setup(oracle_mod, nx, ny, k, quad)
    u = o.initial()
    ug = s.tensor(u)
    ro, rg = o.freeze(u), s.freeze(ug)
    assert abs(ro - rg) <= 1e-14 * ro
    o.set_stage(u, .01)
    s.set_stage(ug, .01)
    up = u + 1e-3 * direction(u.size)
    assert rel(np_(s.residual(s.tensor(up))), o.residual(up)) <= 1e-12
    o.dg_refresh(up)
    s.dg_refresh(s.tensor(up))
    d = direction(u.size, .31, .79)
    assert rel(np_(s.dg_apply(s.tensor(d))), o.dg_apply(d)) <= 1e-12
    for cell in sorted({0, nx * ny // 2, nx * ny - 1}):
        assert rel(s.dg_block(cell, cell), o.dg_block(cell, cell)) <= 1e-12
    o.dg_precond_refresh()
    s.precond_refresh("dg")
    assert rel(np_(s.precond_apply("dg", s.tensor(d))), o.dg_precond_apply(d)) <= 1e-10


@pytest.mark.parametrize("nx,ny,k,quad", CASES[:2])
def test_hdg_condensation(oracle_mod, nx, ny, k, quad):
    o, s = setup(oracle_mod, nx, ny, k, quad)
    u = o.initial()
    o.freeze(u)
    s.freeze(s.tensor(u))
    o.set_stage(u, .01)
    s.set_stage(s.tensor(u), .01)
    up = u + 1e-3 * direction(u.size)
    r = o.residual(up)
    o.hdg_refresh(up, r)
    s.hdg_refresh_projected(s.tensor(up), s.tensor(r))
    assert rel(np_(s.hdg_rhs()), o.hdg_rhs()) <= 1e-11
    dl = direction(o.trace_size)
    assert rel(np_(s.hdg_apply(s.tensor(dl))), o.hdg_apply(dl)) <= 1e-11
    assert rel(np_(s.hdg_recover(s.tensor(dl))), o.hdg_recover(dl)) <= 1e-11


def test_admissibility_at_the_volume_points(oracle_mod):
    """Positive at the nodes and faces, negative between them: only the over-integrated rule
    rejects it, on the device as in the oracle."""
    from dg_hdg_euler_cpp_b200.solver import Solver

    o = oracle_mod.Oracle("--nx 3 --ny 3 --k 3 --quad 8")
    s = Solver(nx=3, ny=3, k=3, quad=8, method="dg")
    sc = Solver(nx=3, ny=3, k=3, method="dg")
    u = o.initial()
    bad = u.copy()
    plane = 16
    bad[0:plane] = np.tile([1., 1e-3, 1e-3, 1.], 4)
    bad[plane:3 * plane] = 0.
    bad[3 * plane:4 * plane] = 1.
    assert sc.admissible(sc.tensor(bad))
    assert not s.admissible(s.tensor(bad)) and not o.admissible(bad)
    assert s.admissible(s.tensor(u))


@pytest.mark.parametrize("method", ["dg", "hdg"])
def test_advance_matches_oracle(oracle_mod, method):
    """TimeIntegrator::advance with Q = k + 3 on a 4x4 k = 2 mesh, BE then DIRK3."""
    from dg_hdg_euler_cpp_b200.solver import Solver

    for integrator in ("be", "ssp-dirk3"):
        args = f"--nx 4 --ny 4 --k 2 --quad 5 --cfl 2 --integrator {integrator} --T 0.02 --restart 20"
        o = oracle_mod.Oracle(args)
        u0 = o.initial()
        so, st_o, _ = o.advance(method, u0)
        s = Solver(nx=4, ny=4, k=2, quad=5, cfl=2.0, integrator=integrator, final_time=0.02, restart=20,
                   method=method)
        sg, st_g, _ = s.advance(method, u0)
        assert np.max(np.abs(sg - so)) <= 1e-10 * np.max(np.abs(so)), integrator
        assert st_g["newton_iterations"] == st_o["newton_iterations"]
        assert abs(st_g["krylov_iterations"] - st_o["krylov_iterations"]) <= 2 * st_o["newton_iterations"]
        s.close()


def test_mixed_precision_matches_fp64():
    from dg_hdg_euler_cpp_b200.solver import Solver

    out = {}
    for precision in ("fp64", "mixed"):
        s = Solver(nx=4, ny=4, k=2, quad=5, cfl=2.0, integrator="be", final_time=0.02, restart=20,
                   method="dg", precision=precision)
        out[precision] = s.advance("dg", np_(s.initial()))[0]
        s.close()
    assert np.max(np.abs(out["mixed"] - out["fp64"])) <= 1e-10 * np.max(np.abs(out["fp64"]))


@pytest.mark.parametrize("nx,ny,k,quad", CASES)
def test_adjoint_apply_and_transposed_solve(oracle_mod, nx, ny, k, quad):
    """J^T w with the over-integrated volume term: the transpose identity, the transpose of the
    oracle's coupling blocks, and the transposed block-Jacobi solve with those blocks."""
    o, s = setup(oracle_mod, nx, ny, k, quad)
    u = o.initial()
    o.freeze(u)
    s.freeze(s.tensor(u))
    o.set_stage(u, .004)
    s.set_stage(s.tensor(u), .004)
    up = u + 1e-3 * direction(u.size)
    o.dg_refresh(up)
    s.dg_refresh(s.tensor(up))
    v, w = direction(u.size, .31, .79), direction(u.size, .17, .53)
    jv = np_(s.dg_apply(s.tensor(v)))
    jtw = np_(s.dg_apply_T(s.tensor(w)))
    lhs, rhs = float(jtw @ v), float(w @ jv)
    assert abs(lhs - rhs) <= 1e-12 * max(abs(lhs), np.linalg.norm(jtw) * np.linalg.norm(v))
    ref = o.dg_apply_transpose(w)
    assert rel(jtw, ref) <= 1e-12
    s.precond_refresh("dg")
    z = np_(s.precond_apply("dg_t", s.tensor(v)))
    m = o.block
    for cell in sorted({0, nx * ny // 2, nx * ny - 1}):
        x = np.linalg.solve(o.dg_block(cell, cell).T, v[cell * m:(cell + 1) * m])
        assert rel(z[cell * m:(cell + 1) * m], x) <= 1e-10


def test_discrete_adjoint_gradient_with_quadrature():
    """DIRK3 discrete adjoint on an over-integrated run against central differences (h = 1e-6)
    of the replayed trajectory, as for the collocated rule."""
    import ctypes

    from dg_hdg_euler_cpp_b200 import _lib
    from dg_hdg_euler_cpp_b200.solver import Integrator, Solver

    nx, ny, k, steps, every = 6, 6, 3, 3, 2
    s = Solver(nx=nx, ny=ny, k=k, quad=6, cfl=0.3, integrator="ssp-dirk3", steps=steps, method="dg", restart=20)
    it = Integrator(s, "dg")
    u0 = np_(s.initial())
    n = s.size
    rho = ((np.arange(n) // (k + 1) ** 2) % 4) == 0
    grad = np.zeros(n)
    st = _lib.dgh_adjoint_stats()
    rc = s.lib.dgh_dirk3_adjoint(it.h, steps, every, u0.ctypes.data_as(ctypes.c_void_p),
                                 grad.ctypes.data_as(ctypes.c_void_p), ctypes.byref(st))
    assert rc == 0, s.lib.dgh_integrator_error(it.h).decode()

    def objective(u):
        val = ctypes.c_double()
        rc = s.lib.dgh_dirk3_replay(it.h, np.ascontiguousarray(u).ctypes.data_as(ctypes.c_void_p), ctypes.byref(val))
        assert rc == 0, s.lib.dgh_integrator_error(it.h).decode()
        return val.value

    h = 1e-6
    for seed in range(2):
        phi = np.where(rho, np.random.default_rng(seed).standard_normal(n), 0.0) * 0.05 * np.abs(u0)
        fd = (objective(u0 + h * phi) - objective(u0 - h * phi)) / (2 * h)
        ad = float(grad @ phi)
        assert abs(fd - ad) <= 1e-6 * abs(ad), (seed, fd, ad)
    it.close()
    s.close()


def test_cli_quad_summary_and_history(oracle_mod):
    """dg_hdg_2d --quad 5 on 4x4 k = 2 through the CLI: the summary reports the volume rule's
    point count, and the Newton history of each method follows the oracle's advance."""
    import subprocess
    import tempfile

    from conftest import assert_history_close, read_csv
    from dg_hdg_euler_cpp_b200 import BIN_PATH

    args = "--nx 4 --ny 4 --k 2 --quad 5 --cfl 2 --integrator be --T 0.02 --restart 20"
    with tempfile.TemporaryDirectory() as tmp:
        res = subprocess.run([str(BIN_PATH), *args.split(), "--method", "both", "--no-save-solution",
                              "--prefix", f"{tmp}/run"], capture_output=True, text=True, timeout=600)
        assert res.returncode == 0, res.stderr + res.stdout
        summ = read_csv(f"{tmp}/run_summary.csv")
        rows = read_csv(f"{tmp}/run_iterations.csv")
    o = oracle_mod.Oracle(args)
    for row in summ:
        assert row["quad"] == "5"
        _, st, ups = o.advance(row["method"], o.initial())
        assert int(row["newton_iterations"]) == st["newton_iterations"]
        ours = [r for r in rows if r["method"] == row["method"]]
        # oracle update rows: step, stage, iteration, krylov, time, stage_time, dt, cfl, rms, ...
        ref = [dict(method=row["method"], step=str(int(u[0])), stage=str(int(u[1])), iteration=str(int(u[2])),
                    krylov_iterations=int(u[3]), time=u[4], stage_time=u[5], dt=u[6], cfl=u[7],
                    residual_physical_rms=u[8]) for u in ups]
        assert_history_close(ours, ref, krylov_slack=2)
