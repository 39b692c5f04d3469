"""GPU kernels against the CPU oracle on the same inputs (FP64 unless stated).

Tolerances: residual, J*v, blocks and norms agree to 1e-12 relative (different summation
order only); the preconditioner solve to 1e-10 (FP64 LU, conditioning ~1e2) or 1e-4 (FP32
factors); GMRES solutions to 1e-9 relative since both solve to ltol = 1e-12.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CASES = [(4, 4, 2), (5, 3, 1), (3, 4, 4), (3, 3, 8), (6, 5, 0), (4, 3, 3)]


def direction(n):
    i = np.arange(n)
    return .2 * np.sin(.31 * i) + .1 * np.cos(.79 * i)  # check_2d.cpp:9-11


def rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def setup_pair(oracle_mod, nx, ny, k, precision="fp64", **kw):
    from dg_hdg_euler_cpp_b200.solver import Solver

    args = f"--nx {nx} --ny {ny} --k {k} --cfl 2 --integrator be --steps 1"
    o = oracle_mod.Oracle(args)
    s = Solver(nx=nx, ny=ny, k=k, cfl=2.0, integrator="be", steps=1, method="both", precision=precision, **kw)
    return o, s


def np_(t):
    return t.detach().cpu().numpy()


@pytest.mark.parametrize("nx,ny,k", CASES)
def test_initial_freeze_residual(oracle_mod, nx, ny, k):
    o, s = setup_pair(oracle_mod, nx, ny, k)
    uo = o.initial()
    ug = s.initial()
    assert rel(np_(ug), uo) <= 1e-13
    ug = s.tensor(uo)  # continue from identical inputs
    rate_o = o.freeze(uo)
    rate_g = s.freeze(ug)
    assert abs(rate_o - rate_g) <= 1e-14 * rate_o
    assert rel(s.speeds(), o.speeds()) <= 1e-14
    dt = .003
    o.set_stage(uo, dt)
    s.set_stage(ug, dt)
    up = uo + 1e-3 * direction(uo.size)
    ro = o.residual(up)
    rg = np_(s.residual(s.tensor(up)))
    assert rel(rg, ro) <= 1e-12
    assert abs(s.dual_norm(s.tensor(ro)) - o.dual_norm(ro)) <= 1e-13 * o.dual_norm(ro)
    assert s.admissible(s.tensor(up)) == o.admissible(up) == True  # noqa: E712
    bad = up.copy()
    bad[0] = -1.0  # negative density at a node
    assert s.admissible(s.tensor(bad)) is False and o.admissible(bad) is False
    bad = up.copy()
    bad[3] = np.nan
    assert s.admissible(s.tensor(bad)) is False and o.admissible(bad) is False
    assert rel(s.integral(s.tensor(up)), o.integral(up)) <= 1e-13
    if k >= 1:
        lam_o = o.trace(up)
        assert rel(np_(s.trace(s.tensor(up))), lam_o) <= 1e-13


@pytest.mark.parametrize("nx,ny,k", CASES)
def test_dg_jv_blocks_and_precond(oracle_mod, nx, ny, k):
    o, s = setup_pair(oracle_mod, nx, ny, k)
    uo = o.initial()
    ug = s.tensor(uo)
    o.freeze(uo)
    s.freeze(ug)
    o.set_stage(uo, .003)
    s.set_stage(ug, .003)
    o.dg_refresh(uo)
    s.dg_refresh(ug)
    d = direction(uo.size)
    jo = o.dg_apply(d)
    jg = np_(s.dg_apply(s.tensor(d)))
    assert rel(jg, jo) <= 1e-12
    for cell in sorted({0, o.cells // 2, o.cells - 1}):
        bo = o.dg_block(cell, cell)
        bg = s.dg_block(cell, cell)
        assert rel(bg, bo) <= 1e-13
    o.dg_precond_refresh()
    s.precond_refresh("dg")
    zo = o.dg_precond_apply(d)
    zg = np_(s.precond_apply("dg", s.tensor(d)))
    assert rel(zg, zo) <= 1e-10


@pytest.mark.parametrize("nx,ny,k", [(4, 4, 2), (3, 4, 4), (3, 3, 8)])
def test_mixed_precision_precond(oracle_mod, nx, ny, k):
    o, s = setup_pair(oracle_mod, nx, ny, k, precision="mixed")
    uo = o.initial()
    ug = s.tensor(uo)
    o.freeze(uo)
    s.freeze(ug)
    o.set_stage(uo, .003)
    s.set_stage(ug, .003)
    o.dg_refresh(uo)
    s.dg_refresh(ug)
    o.dg_precond_refresh()
    s.precond_refresh("dg")
    d = direction(uo.size)
    zo = o.dg_precond_apply(d)
    zg = np_(s.precond_apply("dg", s.tensor(d)))
    assert rel(zg, zo) <= 1e-4


@pytest.mark.parametrize("nx,ny,k", [(4, 4, 2), (3, 4, 4), (3, 3, 8)])
def test_mixed_precision_hdg_face_precond(oracle_mod, nx, ny, k):
    """FP32 face-block factors (warp-per-block LU) against the oracle's FP64 block Jacobi."""
    o, s = setup_pair(oracle_mod, nx, ny, k, precision="mixed")
    uo = o.initial()
    ug = s.tensor(uo)
    o.freeze(uo)
    s.freeze(ug)
    o.set_stage(uo, .003)
    s.set_stage(ug, .003)
    r = o.residual(uo)
    o.hdg_refresh(uo, r)
    s.hdg_refresh_projected(ug, s.tensor(r))
    o.hdg_precond_refresh()
    s.precond_refresh("hdg")
    dl = direction(o.trace_size)
    assert rel(np_(s.precond_apply("hdg", s.tensor(dl))), o.hdg_precond_apply(dl)) <= 1e-4


@pytest.mark.parametrize("nx,ny,k", CASES)
def test_hdg_condensation_schur_recovery(oracle_mod, nx, ny, k):
    o, s = setup_pair(oracle_mod, nx, ny, k)
    uo = o.initial()
    ug = s.tensor(uo)
    o.freeze(uo)
    s.freeze(ug)
    o.set_stage(uo, .003)
    s.set_stage(ug, .003)
    up = uo + 1e-3 * direction(uo.size)
    r = o.residual(up)
    o.hdg_refresh(up, r)
    s.hdg_refresh_projected(s.tensor(up), s.tensor(r))
    assert rel(np_(s.hdg_rhs()), o.hdg_rhs()) <= 1e-11
    dl = direction(o.trace_size)
    assert rel(np_(s.hdg_apply(s.tensor(dl))), o.hdg_apply(dl)) <= 1e-11
    for face in sorted({0, o.cells - 1, o.cells, o.faces - 1}):
        assert rel(s.hdg_block(face, face), o.hdg_block(face, face)) <= 1e-11
    assert rel(np_(s.hdg_recover(s.tensor(dl))), o.hdg_recover(dl)) <= 1e-11
    assert rel(np_(s.hdg_recovered_residual(s.tensor(dl))), o.hdg_recovered_residual(dl)) <= 1e-12
    o.hdg_precond_refresh()
    s.precond_refresh("hdg")
    assert rel(np_(s.precond_apply("hdg", s.tensor(dl))), o.hdg_precond_apply(dl)) <= 1e-10


@pytest.mark.parametrize("nx,ny,k", [(4, 4, 2), (3, 4, 4), (3, 3, 8)])
def test_gmres_dg_and_hdg(oracle_mod, nx, ny, k):
    o, s = setup_pair(oracle_mod, nx, ny, k, restart=20)
    uo = o.initial()
    ug = s.tensor(uo)
    o.freeze(uo)
    s.freeze(ug)
    dt = 5.0 / o.freeze(uo)
    s.freeze(ug)
    o.set_stage(uo, dt)
    s.set_stage(ug, dt)
    up = uo + 1e-3 * direction(uo.size)
    r = o.residual(up)
    o.dg_refresh(up)
    s.dg_refresh(s.tensor(up))
    o.dg_precond_refresh()
    s.precond_refresh("dg")
    xo, ito, relo, _ = o.gmres(0, -r, 20, 1500, 1e-12)
    xg, itg, relg, resg = s.gmres("dg", s.tensor(-r), 1500, 1e-12)
    assert abs(ito - itg) <= 1
    assert relg <= 1e-12
    assert rel(np_(xg), xo) <= 1e-9
    # the true residual returned equals rhs - J x
    jx = o.dg_apply(np_(xg))
    assert np.max(np.abs(np_(resg) - (-r - jx))) <= 1e-11 * np.max(np.abs(r))
    o.hdg_refresh(up, r)
    s.hdg_refresh_projected(s.tensor(up), s.tensor(r))
    o.hdg_precond_refresh()
    s.precond_refresh("hdg")
    rhs = o.hdg_rhs()
    lo, ito, relo, _ = o.gmres(1, rhs, 20, 1500, 1e-12)
    lg, itg, relg, _ = s.gmres("hdg", s.tensor(rhs), 1500, 1e-12)
    assert abs(ito - itg) <= 1
    assert rel(np_(lg), lo) <= 1e-9
