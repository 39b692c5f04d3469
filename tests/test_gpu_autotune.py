"""Per-degree autotuner (dgh_config.autotune, dgh_autotune_report): the factorisation variants it
chooses between compute the same factors up to rounding, so tuned Newton updates agree with the
untuned ones to the linear tolerance; the choice is reported and cached per (degree, precision)."""
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
    assert rep0["dg_variant"] == 0 and rep0["hdg_variant"] == 0
    assert rep1["dg_variant"] in (0, 1) and rep1["hdg_variant"] in (0, 1)
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
    assert second["tune_ms"] == {"dg": [0.0, 0.0], "hdg": [0.0, 0.0]}
    assert second["dg_variant"] == first["dg_variant"] and second["hdg_variant"] == first["hdg_variant"]


def test_report_before_factor_and_1d():
    from dg_hdg_euler_cpp_b200.solver import Solver

    s = Solver(nx=4, ny=4, k=3, autotune=1)
    assert s.autotune_report()["dg_variant"] == -1
    s.close()
    s = Solver(dim=1, cells=16, k=3, autotune=1)
    assert s.autotune_report() == {"dg_variant": -1, "hdg_variant": -1,
                                   "tune_ms": {"dg": [0.0, 0.0], "hdg": [0.0, 0.0]}}
    s.close()
