"""The oracle's over-integrated 2D volume terms (--quad Q > k+1: tensor_product.cpp:11-21,57-72,
volume_jacobian.cpp:90-116, discretization.cpp:111-122,184-192,219-233).  No archived run uses
them, so they are pinned by their own mathematics: J*v is the derivative of R (central
differences with the speeds frozen), the assembled blocks reproduce J*v, the interpolation and
the weak form at Q points reduce to the collocated ones for Q = n, and a higher rule changes R
only at the size of the quadrature error."""
import sys

import numpy as np
import pytest

from conftest import ROOT

sys.path.insert(0, str(ROOT / "oracle"))


def setup(nx, ny, k, quad, step=.01):
    import oracle_py

    o = oracle_py.Oracle(f"--nx {nx} --ny {ny} --k {k} --quad {quad} --integrator be --steps 1")
    u = o.initial()
    o.freeze(u)
    o.set_stage(u, step)
    return o, u


def direction(n, a=.37, b=1.3):
    i = np.arange(n)
    return np.sin(a * i) + .3 * np.cos(b * i)


@pytest.mark.parametrize("nx,ny,k,quad", [(3, 4, 2, 4), (4, 3, 3, 6), (3, 3, 1, 3)])
def test_jv_is_the_derivative_of_the_residual(nx, ny, k, quad):
    o, u = setup(nx, ny, k, quad)
    up = u + 1e-3 * direction(u.size, .11, .7)
    o.dg_refresh(up)
    d = direction(u.size)
    eps = 1e-6
    fd = (o.residual(up + eps * d) - o.residual(up - eps * d)) / (2 * eps)
    jv = o.dg_apply(d)
    assert np.max(np.abs(jv - fd)) <= 1e-6 * np.max(np.abs(jv))


@pytest.mark.parametrize("nx,ny,k,quad", [(3, 3, 2, 5), (3, 4, 3, 5)])
def test_blocks_reproduce_jv(nx, ny, k, quad):
    o, u = setup(nx, ny, k, quad)
    o.dg_refresh(u)
    m = 4 * (k + 1) ** 2
    d = np.zeros(u.size)
    d[m:2 * m] = direction(m)  # cell 1 only
    jv = o.dg_apply(d)
    for row in range(nx * ny):
        if row == 1 or np.max(np.abs(jv[row * m:(row + 1) * m])) > 0:
            blk = o.dg_block(row, 1)
            got = blk @ d[m:2 * m]
            assert np.max(np.abs(got - jv[row * m:(row + 1) * m])) <= 1e-12 * np.max(np.abs(jv))


@pytest.mark.parametrize("nx,ny,k,quad", [(3, 3, 2, 5), (3, 4, 1, 4)])
def test_transpose_identity(nx, ny, k, quad):
    """The adjoint restated from the coupling blocks is the transpose of the matrix-free J*v."""
    o, u = setup(nx, ny, k, quad)
    o.dg_refresh(u + 1e-3 * direction(u.size, .2, .9))
    v, w = direction(u.size), direction(u.size, .17, .53)
    lhs, rhs = float(o.dg_apply_transpose(w) @ v), float(w @ o.dg_apply(v))
    assert abs(lhs - rhs) <= 1e-12 * max(abs(rhs), 1.0)


def test_rule_of_n_points_is_the_collocated_one():
    a, u = setup(4, 3, 3, 0)
    b, _ = setup(4, 3, 3, 4)
    up = u + 1e-3 * direction(u.size)
    assert np.max(np.abs(a.residual(up) - b.residual(up))) <= 1e-13 * np.max(np.abs(a.residual(up)))


def test_higher_rules_converge():
    """R with Q = n+1, n+3, n+5 points: the differences shrink as the rule grows (the flux is
    smooth but not polynomial)."""
    k = 3
    res = {}
    for quad in (k + 2, k + 4, k + 6):
        o, u = setup(4, 4, k, quad)
        res[quad] = o.residual(u + 1e-3 * direction(u.size))
    d1 = np.max(np.abs(res[k + 4] - res[k + 2]))
    d2 = np.max(np.abs(res[k + 6] - res[k + 4]))
    assert d2 < 0.5 * d1


def test_admissibility_checks_the_volume_points():
    """A cell whose density is positive at the nodes and on the faces but negative between the
    nodes (nodal values 1, 1e-3, 1e-3, 1 along x at k = 3) fails only with the over-integrated
    rule, which also checks the volume points."""
    o_c, u = setup(3, 3, 3, 0)
    o_q, _ = setup(3, 3, 3, 8)
    assert o_c.admissible(u) and o_q.admissible(u)
    bad = u.copy()
    plane = 16
    f = np.array([1., 1e-3, 1e-3, 1.])
    bad[0:plane] = np.tile(f, 4)       # rho(ix, iy) = f(ix)
    bad[plane:3 * plane] = 0.          # no momentum
    bad[3 * plane:4 * plane] = 1.      # pressure 2 at the nodes and faces
    assert o_c.admissible(bad)
    assert not o_q.admissible(bad)


def test_dg_and_hdg_runs_agree():
    """The HDG condensation uses the over-integrated cell block, the DG path the over-integrated
    residual and J*v: both runs reach the same states (and differ from the collocated run at
    the size of the quadrature aliasing)."""
    import oracle_py

    o = oracle_py.Oracle("--nx 4 --ny 4 --k 2 --quad 5 --cfl 2 --integrator ssp-dirk3 --T 0.02 --restart 20")
    u0 = o.initial()
    a, _, _ = o.advance("dg", u0)
    b, _, _ = o.advance("hdg", u0)
    assert np.max(np.abs(a - b)) <= 1e-12 * np.max(np.abs(a))
    c, _, _ = oracle_py.Oracle("--nx 4 --ny 4 --k 2 --cfl 2 --integrator ssp-dirk3 --T 0.02 --restart 20").advance("dg", u0)
    assert np.max(np.abs(a - c)) > 1e-6 * np.max(np.abs(a))
