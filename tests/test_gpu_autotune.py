"""Per-degree autotuner (dgh_config.autotune, dgh_autotune_report, dgh_autotune_shapes): the
factorisation variants it chooses between compute the same factors up to rounding, so tuned
Newton updates agree with the untuned ones to the linear tolerance; the launch shapes (the DG
block solve's grid, the fused factorisation's CTAs per SM) give bitwise-equal results; the
choices are reported and cached per (degree, precision) (and cell count for the solve grid)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def run_updates(autotune, precision, kw, count=3):
    """Rows of `count` BE updates per method, the final states, and the tuner's report."""
    import ctypes

    from dg_hdg_euler_cpp_b200.solver import Integrator, Solver

    s = Solver(cfl=5.0, integrator="be", steps=1, newton_steps=count, method="both", restart=20,
               precision=precision, autotune=autotune, **kw)
    rows, states = {}, {}
    for method in ("dg", "hdg"):
        it = Integrator(s, method)
        it.stage_begin(s.initial())
        rows[method] = [it.update() for _ in range(count)]
        state = s.vec()
        p = ctypes.c_void_p(it.state_ptr())
        s._rc(s.lib.dgh_axpby(s.h, 1.0, p, 0.0, p, ctypes.c_void_p(state.data_ptr()), state.numel()))
        s._rc(s.lib.dgh_sync(s.h))
        states[method] = state.cpu().numpy()
        it.close()
    report = s.autotune_report()
    s.close()
    return rows, states, report


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("k", [2, 5])
def test_tuned_updates_match_default(precision, k):
    kw = dict(nx=8, ny=8, k=k)
    base, u0, rep0 = run_updates(0, precision, kw)
    tuned, u1, rep1 = run_updates(1, precision, kw)
    assert rep0["dg_variant"] == 0 and rep0["hdg_variant"] == 0 and rep0["solve_shape"] == 0
    assert rep0["fused_ctas"] == 2 and rep1["fused_ctas"] in (1, 2)
    assert rep1["dg_variant"] in (0, 1) and rep1["hdg_variant"] in (0, 1) and rep1["solve_shape"] in (0, 1)
    for method in ("dg", "hdg"):
        # three Newton updates solved to the linear tolerance 1e-12: the states agree far below
        # the update size whichever factorisation preconditioned the solves
        assert np.max(np.abs(u1[method] - u0[method])) <= 1e-9 * np.max(np.abs(u0[method]))
        for a, b in zip(base[method], tuned[method]):
            assert abs(b["krylov_iterations"] - a["krylov_iterations"]) <= max(2, a["krylov_iterations"] // 10)


def test_choice_cached_per_degree():
    """The first context of a (degree, precision) times both variants on its own cells; a second
    context of the same degree and precision reuses the cached choice without timing."""
    kw = dict(nx=6, ny=6, k=7)
    _, _, first = run_updates(1, "fp64", kw, count=1)
    _, _, second = run_updates(1, "fp64", kw, count=1)
    assert all(t > 0 for t in first["tune_ms"]["dg"] + first["tune_ms"]["hdg"]) or \
        all(t == 0 for t in first["tune_ms"]["dg"])  # cached by an earlier test of the same degree
    assert second["tune_ms"] == {"dg": [0.0, 0.0], "hdg": [0.0, 0.0]} and second["solve_ms"] == [0.0, 0.0]
    assert second["dg_variant"] == first["dg_variant"] and second["hdg_variant"] == first["hdg_variant"]
    assert second["solve_shape"] == first["solve_shape"] and second["fused_ctas"] == first["fused_ctas"]


def test_report_before_factor_and_1d():
    from dg_hdg_euler_cpp_b200.solver import Solver

    s = Solver(nx=4, ny=4, k=3, autotune=1)
    assert s.autotune_report()["dg_variant"] == -1
    s.close()
    s = Solver(dim=1, cells=16, k=3, autotune=1)
    assert s.autotune_report() == {"dg_variant": -1, "hdg_variant": -1,
                                   "tune_ms": {"dg": [0.0, 0.0], "hdg": [0.0, 0.0]},
                                   "solve_shape": -1, "solve_ms": [0.0, 0.0], "fused_ctas": -1, "fused_ms": [0.0, 0.0]}
    s.close()


@pytest.mark.parametrize("precision,nx,k", [("fp64", 72, 3), ("mixed", 9, 8), ("mixed16", 80, 2), ("mixed", 90, 2)])
def test_solve_shapes_bitwise_equal(oracle_mod, precision, nx, k):
    """Both grid shapes of the DG block solve give bitwise-equal results (each block's solve is
    the same arithmetic whichever warp runs it), and match the oracle's block Jacobi.  The larger
    meshes have more blocks than one round of resident warps, so the two shapes' grids differ."""
    from dg_hdg_euler_cpp_b200.solver import Solver

    o = oracle_mod.Oracle(f"--nx {nx} --ny {nx} --k {k} --cfl 2 --integrator be --steps 1")
    s = Solver(nx=nx, ny=nx, k=k, cfl=2.0, integrator="be", steps=1, method="dg", precision=precision)
    u = o.initial()
    o.freeze(u)
    s.freeze(s.tensor(u))
    o.set_stage(u, .003)
    s.set_stage(s.tensor(u), .003)
    o.dg_refresh(u)
    s.dg_refresh(s.tensor(u))
    o.dg_precond_refresh()
    s.precond_refresh("dg")
    d = .2 * np.sin(.31 * np.arange(o.size)) + .1 * np.cos(.79 * np.arange(o.size))
    out = []
    for shape in (0, 1):
        s.solve_shape(shape)
        out.append(s.precond_apply("dg", s.tensor(d)).cpu().numpy())
    assert np.array_equal(out[0], out[1])
    ref = o.dg_precond_apply(d)
    tol = {"fp64": 1e-10, "mixed": 1e-4, "mixed16": 5e-3}[precision]
    assert np.max(np.abs(out[0] - ref)) <= tol * np.max(np.abs(ref))
    s.close()


@pytest.mark.parametrize("precision,nx,k", [("mixed", 20, 8), ("mixed16", 20, 8), ("mixed16", 40, 3)])
def test_fused_factorisation_residency_bitwise_equal(precision, nx, k):
    """The fused reduced-precision DG factorisation gives bitwise-equal factors with 1 or 2 CTAs
    per SM (each cell is factored by the same arithmetic whichever CTA takes it): the block
    solves agree bitwise."""
    from dg_hdg_euler_cpp_b200.solver import Solver

    outs = []
    for ctas in (1, 2):
        s = Solver(nx=nx, ny=nx, k=k, cfl=2.0, integrator="be", steps=1, method="dg", precision=precision)
        u = s.initial()
        s.freeze(u)
        s.set_stage(u, .003)
        s.dg_refresh(u)
        s.fused_ctas(ctas)
        s.precond_refresh("dg")
        n = u.numel()
        d = .2 * np.sin(.31 * np.arange(n)) + .1 * np.cos(.79 * np.arange(n))
        outs.append(s.precond_apply("dg", s.tensor(d)).cpu().numpy())
        s.close()
    assert np.array_equal(outs[0], outs[1])
