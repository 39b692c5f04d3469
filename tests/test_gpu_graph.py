"""GMRES restart cycles replayed as CUDA graphs (dgh_gmres_graph_enable) against the same cycles
launched step by step: the kernels are the same, so solutions, residuals and iteration counts
must agree bitwise; both agree with the oracle's GMRES to the solve tolerance."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def direction(n):
    i = np.arange(n)
    return .2 * np.sin(.31 * i) + .1 * np.cos(.79 * i)


def np_(t):
    return t.detach().cpu().numpy()


def solve_both(s, op, rhs, limit=1500, tol=1e-12):
    out = []
    for graph in (False, True):
        s.gmres_graph(graph)
        x, it, rel, res = s.gmres(op, s.tensor(rhs), limit, tol)
        out.append((np_(x), it, rel, np_(res)))
    s.gmres_graph(False)
    return out


@pytest.mark.parametrize("nx,k,restart", [(4, 2, 20), (5, 3, 7), (3, 8, 20)])
def test_graph_cycles_equal_stepped_cycles_2d(oracle_mod, nx, k, restart):
    from dg_hdg_euler_cpp_b200.solver import Solver

    o = oracle_mod.Oracle(f"--nx {nx} --ny {nx} --k {k} --cfl 2 --integrator be --steps 1 --restart {restart}")
    s = Solver(nx=nx, ny=nx, k=k, cfl=2.0, integrator="be", steps=1, method="both", restart=restart)
    u = o.initial()
    dt = 5.0 / o.freeze(u)
    s.freeze(s.tensor(u))
    o.set_stage(u, dt)
    s.set_stage(s.tensor(u), dt)
    up = u + 1e-3 * direction(u.size)
    r = o.residual(up)
    o.dg_refresh(up)
    s.dg_refresh(s.tensor(up))
    o.dg_precond_refresh()
    s.precond_refresh("dg")
    (xa, ita, rela, resa), (xb, itb, relb, resb) = solve_both(s, "dg", -r)
    assert ita == itb and rela == relb
    assert np.array_equal(xa, xb) and np.array_equal(resa, resb)
    xo, ito, _, _ = o.gmres(0, -r, restart, 1500, 1e-12)
    assert abs(ito - ita) <= 1 and np.max(np.abs(xa - xo)) <= 1e-9 * np.max(np.abs(xo))
    o.hdg_refresh(up, r)
    s.hdg_refresh_projected(s.tensor(up), s.tensor(r))
    o.hdg_precond_refresh()
    s.precond_refresh("hdg")
    rhs = o.hdg_rhs()
    (la, ita, _, _), (lb, itb, _, _) = solve_both(s, "hdg", rhs)
    assert ita == itb and np.array_equal(la, lb)
    lo, ito, _, _ = o.gmres(1, rhs, restart, 1500, 1e-12)
    assert abs(ito - ita) <= 1 and np.max(np.abs(la - lo)) <= 1e-9 * np.max(np.abs(lo))
    s.close()


def test_graph_limit_and_zero_rhs():
    """The iteration limit inside a cycle and the zero right-hand side behave as in the
    reference (gmres.cpp:21-22, 85): same error, same count, zero solution."""
    from dg_hdg_euler_cpp_b200.solver import DGHError, Solver

    s = Solver(nx=4, ny=4, k=3, cfl=2.0, integrator="be", steps=1, method="dg", restart=10)
    u = s.initial()
    s.freeze(u)
    s.set_stage(u, .05)
    s.dg_refresh(u)
    s.precond_refresh("dg")
    for graph in (False, True):
        s.gmres_graph(graph)
        x, it, rel, _ = s.gmres("dg", s.vec(), 100, 1e-12)
        assert it == 0 and rel == 0 and not np_(x).any()
        with pytest.raises(DGHError, match="GMRES iteration limit reached"):
            s.gmres("dg", s.tensor(direction(s.size)), 13, 1e-14)
    s.close()


def test_graph_newton_updates_equal_stepped_1d_and_2d():
    """Whole Newton updates (integrator) with graph cycles equal the stepped ones bitwise."""
    from dg_hdg_euler_cpp_b200.solver import Integrator, Solver

    for kw in (dict(nx=6, ny=6, k=3), dict(dim=1, cells=24, k=4)):
        rows = {}
        for graph in (False, True):
            s = Solver(cfl=5.0, integrator="be", steps=1, newton_steps=3, method="both", restart=20, **kw)
            s.gmres_graph(graph)
            for method in ("dg", "hdg"):
                it = Integrator(s, method)
                it.stage_begin(s.initial())
                rows[(graph, method)] = [it.update() for _ in range(3)]
                it.close()
            s.close()
        for method in ("dg", "hdg"):
            for a, b in zip(rows[(False, method)], rows[(True, method)]):
                for key in ("residual_physical_rms", "krylov_iterations", "linear_relative_residual", "damping"):
                    assert a[key] == b[key], (kw, method, key)


def test_graph_newton_updates_equal_stepped_1d_block_ilu0():
    """With the 1D block ILU(0) preconditioner (single-CTA sweeps inside the replayed cycles)
    the graph-replayed updates equal the stepped ones bitwise."""
    from dg_hdg_euler_cpp_b200.solver import Integrator, Solver

    rows = {}
    for graph in (False, True):
        s = Solver(dim=1, cells=24, k=3, cfl=5.0, integrator="be", steps=1, newton_steps=3, method="both",
                   restart=20, precond="block-ilu0")
        s.gmres_graph(graph)
        for method in ("dg", "hdg"):
            it = Integrator(s, method)
            it.stage_begin(s.initial())
            rows[(graph, method)] = [it.update() for _ in range(3)]
            it.close()
        s.close()
    for method in ("dg", "hdg"):
        for a, b in zip(rows[(False, method)], rows[(True, method)]):
            for key in ("residual_physical_rms", "krylov_iterations", "linear_relative_residual", "damping"):
                assert a[key] == b[key], (method, key)
