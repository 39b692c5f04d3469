"""The reference's own checks that sit at the LU and integrator boundaries, on the device.

* Forced-pivot block Jacobi (dg_hdg_2d/check/check_2d.cpp:12-25): widths 4, 12, 36 and 324, each
  block a(i, i+1 mod w) = 2 + 0.01 i with a(i, i) += 0.1, so every column's largest entry is off
  the diagonal and every elimination step must pivot; three blocks; ||x - exact|| <= 2e-12 for
  every FP64 LU kernel, and the FP32 factors to FP32 accuracy.
* The pivot sequence with ties: the first largest |a| wins (LAPACK getrf, Eigen PartialPivLU),
  against a plain partial-pivoting restatement in numpy.
* A singular block raises "Singular block Jacobi factor" (block_jacobi.hpp:16-18).
* "Newton line search failed" (time_integrator.cpp:176) and "Recovered DG residual criterion
  failed after Schur refinement" (:149) through the C ABI, reached by lowering the integrator's
  limits (dgh_integrator_set_limits) on ordinary inputs.
* The allocation guard (time_integrator.cpp:7-14): Newton updates allocate no device memory.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def direction(n):
    i = np.arange(n)
    return .2 * np.sin(.31 * i) + .1 * np.cos(.79 * i)


def forced_pivot_block(width):
    a = np.zeros((width, width))
    for i in range(width):
        a[i, (i + 1) % width] = 2. + .01 * i
        a[i, i] += .1
    return a


def variants(width):
    out = [("fp64", 0), ("fp64", 1), ("mixed", 0), ("mixed", 1)]
    if width <= 64:
        out += [("fp64", 2), ("mixed", 2), ("mixed", 3)]
    return out


@pytest.mark.parametrize("width", [4, 12, 36, 324])
def test_forced_pivot_block_jacobi(width):
    from dg_hdg_euler_cpp_b200.solver import BlockJacobi

    blocks = 3
    a = forced_pivot_block(width)
    exact = direction(blocks * width)
    rhs = np.concatenate([a @ exact[i * width:(i + 1) * width] for i in range(blocks)])
    for precision, variant in variants(width):
        bj = BlockJacobi(width, blocks, precision, variant)
        bj.factor(np.stack([a] * blocks))
        x = bj.apply(rhs)
        err = np.linalg.norm(x - exact)
        tol = 2e-12 if precision == "fp64" else 1e-5 * np.linalg.norm(exact)
        assert err <= tol, (width, precision, variant, err)
        if variant != 3:
            # every step pivots: position i holds original row i-1 (mod w) for this pattern
            perm = bj.perm()
            assert all((perm[b] == ref_pivots(a)).all() for b in range(blocks)), (precision, variant)
        bj.close()


def ref_pivots(a):
    """Row partial pivoting with the first largest |a| winning ties; returns the gather
    permutation (position i holds original row perm[i])."""
    a = a.copy()
    n = a.shape[0]
    perm = np.arange(n)
    for k in range(n):
        p = k + int(np.argmax(np.abs(a[k:, k])))  # argmax returns the first of equal maxima
        if p != k:
            a[[k, p]] = a[[p, k]]
            perm[[k, p]] = perm[[p, k]]
        if a[k, k] != 0:
            a[k + 1:, k] /= a[k, k]
            a[k + 1:, k + 1:] -= np.outer(a[k + 1:, k], a[k, k + 1:])
    return perm


@pytest.mark.parametrize("width", [12, 36, 324])
def test_pivot_ties_first_largest_wins(width):
    """Column 0 holds two candidates of equal magnitude and opposite sign (rows 2 and 9, |a| = 4,
    every other entry below 1): the first one must win.  The rest of the block is generic, and
    every kernel's whole permutation equals the first-largest partial-pivoting sequence of a
    numpy restatement; the solves agree."""
    from dg_hdg_euler_cpp_b200.solver import BlockJacobi

    rng = np.random.default_rng(width)
    a = rng.uniform(-1, 1, size=(width, width)) + 2.0 * np.eye(width)
    a[:, 0] = rng.uniform(-.5, .5, size=width)
    a[2, 0], a[9, 0] = -4.0, 4.0
    x0 = direction(width)
    rhs = a @ x0
    expect = ref_pivots(a)
    assert expect[0] == 2
    for precision, variant in variants(width):
        if variant == 3:
            continue
        bj = BlockJacobi(width, 2, precision, variant)
        bj.factor(np.stack([a, a]))
        x = bj.apply(np.concatenate([rhs, rhs]))
        tol = 1e-10 if precision == "fp64" else 1e-4
        assert np.max(np.abs(x[:width] - x0)) <= tol * np.max(np.abs(x0)), (precision, variant)
        perm = bj.perm()[0]
        assert perm[0] == 2, (precision, variant, perm[:4])
        if precision == "fp64":
            assert (perm == expect).all(), (variant, perm[:12], expect[:12])
        bj.close()


@pytest.mark.parametrize("precision,variant", [("fp64", 0), ("fp64", 1), ("fp64", 2), ("mixed", 0), ("mixed", 1),
                                               ("mixed", 2)])
def test_singular_block_raises_reference_message(precision, variant):
    from dg_hdg_euler_cpp_b200.solver import BlockJacobi, DGHError

    a = forced_pivot_block(36)
    a[:, 5] = 0.0  # a zero column: no pivot exists at step 5
    bj = BlockJacobi(36, 2, precision, variant)
    with pytest.raises(DGHError, match="Singular block Jacobi factor") as exc:
        bj.factor(np.stack([forced_pivot_block(36), a]))
    assert exc.value.code == 3
    bj.close()


def _integrator(method, **kw):
    from dg_hdg_euler_cpp_b200.solver import Integrator, Solver

    s = Solver(nx=6, ny=6, k=3, cfl=2.0, integrator="be", steps=1, restart=20, method=method, **kw)
    it = Integrator(s, method)
    it.stage_begin(s.initial())
    return s, it


@pytest.mark.parametrize("method", ["dg", "hdg"])
def test_line_search_failure_message(method):
    from dg_hdg_euler_cpp_b200.solver import DGHError

    s, it = _integrator(method)
    it.set_limits(4, 0)
    with pytest.raises(DGHError, match="^Newton line search failed$") as exc:
        it.update()
    assert exc.value.code == 8
    it.set_limits(4, 30)
    it.stage_begin(s.initial())
    assert it.update()["damping"] > 0  # the same update with the reference's limit succeeds
    it.close()
    s.close()


@pytest.mark.parametrize("condense32", [0, 1])
def test_hdg_schur_attempts_exhausted_message(condense32):
    from dg_hdg_euler_cpp_b200.solver import DGHError

    s, it = _integrator("hdg", precision="mixed", condense32=condense32)
    it.set_limits(0, 30)
    with pytest.raises(DGHError, match="^Recovered DG residual criterion failed after Schur refinement$") as exc:
        it.update()
    assert exc.value.code == 8
    it.close()
    s.close()


@pytest.mark.parametrize("method,precision,condense32", [("dg", "fp64", 0), ("dg", "mixed", 0), ("hdg", "fp64", 0),
                                                         ("hdg", "mixed", 1)])
def test_newton_updates_allocate_no_device_memory(method, precision, condense32):
    """time_integrator.cpp:7-14 forbids allocation inside a Newton update.  After a first update
    (which may build the GMRES cycle graphs), further updates change neither the context's own
    device bytes nor the device's free memory."""
    import torch

    s, it = _integrator(method, precision=precision, condense32=condense32)
    s.gmres_graph(True)
    it.update()
    torch.cuda.synchronize()
    bytes0, free0 = s.device_bytes(), torch.cuda.mem_get_info(s.device)[0]
    for _ in range(3):
        it.update()
    torch.cuda.synchronize()
    assert s.device_bytes() == bytes0
    assert torch.cuda.mem_get_info(s.device)[0] == free0
    it.close()
    s.close()
