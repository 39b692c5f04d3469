"""Lockstep batch of GMRES solves (dgh_batch_lockstep, dgh_lockstep_*): the restart cycles of
members of different degree and mesh size advanced together, every Arnoldi phase one kernel
launch over all of them — DG members (block solve + J·v) and HDG members (face preconditioner +
Schur apply) in groups of their own.  Each member runs its single-problem kernel bodies on its
own buffers with its own block partitions, so its update rows and states equal its single run
bitwise; 1D and other members outside a lockstep class keep solving independently; a member
whose solve fails reports its own error while the others complete."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

COMMON = dict(cfl=5.0, integrator="be", steps=1, restart=30, max_linear=1500)
DG_MEMBERS = [dict(nx=12, ny=9, k=2), dict(nx=7, ny=7, k=8), dict(nx=10, ny=6, k=4), dict(nx=5, ny=8, k=3),
              dict(nx=9, ny=9, k=5), dict(nx=6, ny=6, k=8), dict(nx=16, ny=12, k=1)]
AMPLITUDES = [0.1, 0.2, 0.05, 0.15, 0.12, 0.08, 0.18]
KEYS = ("krylov_iterations", "residual_physical_rms", "linear_relative_residual", "dg_linear_relative_residual",
        "damping", "dt", "cfl")


def start_states(batch, members, amplitudes):
    from dg_hdg_euler_cpp_b200.solver import perturb

    out = []
    for i, (m, a) in enumerate(zip(members, amplitudes)):
        u = batch.initial(i)
        out.append(perturb(u, m["nx"], m["ny"], m["k"], a) if m.get("dim", 2) == 2 else u)
    return out


def single_run(kw, u0, updates):
    from dg_hdg_euler_cpp_b200.solver import Integrator, Solver

    s = Solver(**kw)
    it = Integrator(s, kw["method"])
    dt = it.stage_begin(s.tensor(u0))
    rows = [it.update() for _ in range(updates)]
    state = s.vec()
    p = ctypes.c_void_p(it.state_ptr())
    s._rc(s.lib.dgh_axpby(s.h, 1.0, p, 0.0, p, ctypes.c_void_p(state.data_ptr()), state.numel()))
    s._rc(s.lib.dgh_sync(s.h))
    out = state.cpu().numpy()
    it.close()
    s.close()
    return dt, rows, out


def run_batch(members, amplitudes, updates, lockstep=True, graph=False):
    from dg_hdg_euler_cpp_b200.solver import Batch

    b = Batch(members)
    b.gmres_graph(graph)
    b.lockstep(lockstep)
    u0 = start_states(b, members, amplitudes)
    dts = b.stage_begin(u0)
    rows = [b.update() for _ in range(updates)]
    finals = [b.state(i) for i in range(b.count)]
    report = b.lockstep_report()
    b.close()
    return u0, dts, rows, finals, report


def assert_equal_to_single_runs(members, u0, dts, rows, finals, updates):
    for i, kw in enumerate(members):
        dt, ref_rows, ref_state = single_run(kw, u0[i], updates)
        assert dts[i] == dt, i
        for u in range(updates):
            for key in KEYS:
                assert rows[u][i][key] == ref_rows[u][key], (i, u, key, rows[u][i][key], ref_rows[u][key])
        assert np.array_equal(finals[i], ref_state), i


@pytest.mark.parametrize("precision,graph", [("mixed", False), ("fp64", False), ("mixed16", False), ("mixed", True),
                                             ("fp64", True)])
def test_lockstep_members_equal_single_runs_bitwise(precision, graph):
    """Seven DG members of degrees 1-8 on different meshes, three Newton updates in lockstep,
    the cycles launched step by step or replayed as one CUDA graph per restart cycle (when the
    members replay their own cycles as graphs); the single runs launch theirs step by step."""
    members = [dict(COMMON, method="dg", precision=precision, **m) for m in DG_MEMBERS]
    updates = 3
    u0, dts, rows, finals, report = run_batch(members, AMPLITUDES, updates, graph=graph)
    assert report["sessions"] == updates
    # one group step per Arnoldi step of the member with the most iterations in each update
    longest = sum(max(rows[u][i]["krylov_iterations"] for i in range(len(members))) for u in range(updates))
    assert report["steps"] == longest
    assert_equal_to_single_runs(members, u0, dts, rows, finals, updates)


@pytest.mark.parametrize("precision,condense32,graph", [("mixed", 0, False), ("fp64", 0, False), ("mixed", 1, False),
                                                       ("mixed", 0, True)])
def test_lockstep_hdg_members_equal_single_runs_bitwise(precision, condense32, graph):
    """Six HDG members of degrees 1-8 in lockstep (FP32 face inverses, or FP64 face LU factors;
    with the FP32 condensation the FP32 Schur blocks and, after the first lockstep solve, the
    refinement passes' solves on their own), three Newton updates."""
    members = [dict(COMMON, method="hdg", precision=precision, condense32=condense32, **m) for m in DG_MEMBERS[:6]]
    updates = 3
    u0, dts, rows, finals, report = run_batch(members, AMPLITUDES[:6], updates, graph=graph)
    assert report["sessions"] == updates and report["steps"] > 0
    assert_equal_to_single_runs(members, u0, dts, rows, finals, updates)


def test_lockstep_leaves_other_members_independent():
    """DG members in two lockstep classes (two precisions) and an HDG member in a third, beside 1D
    and over-integrated DG members, which keep solving on their own; everything equals the single
    runs bitwise."""
    members = [dict(COMMON, method="dg", precision="mixed", **DG_MEMBERS[0]),
               dict(COMMON, method="hdg", precision="mixed", nx=6, ny=5, k=3),
               dict(COMMON, method="dg", precision="fp64", **DG_MEMBERS[2]),
               dict(COMMON, method="dg", precision="mixed", **DG_MEMBERS[1]),
               dict(COMMON, method="dg", precision="fp64", nx=5, ny=5, k=2, quad=5),
               dict(COMMON, method="dg", dim=1, cells=40, k=2),
               dict(COMMON, method="dg", precision="fp64", **DG_MEMBERS[3])]
    amplitudes = [0.1, 0.2, 0.05, 0.15, 0.1, 0.0, 0.12]
    u0, dts, rows, finals, report = run_batch(members, amplitudes, 2)
    assert report["sessions"] == 3 * 2  # three groups (DG mixed, DG fp64, HDG mixed), two updates
    assert_equal_to_single_runs(members, u0, dts, rows, finals, 2)


def test_lockstep_matches_independent_batch():
    members = [dict(COMMON, method="dg", precision="mixed", **m) for m in DG_MEMBERS[:4]]
    a = run_batch(members, AMPLITUDES[:4], 2, lockstep=True)
    b = run_batch(members, AMPLITUDES[:4], 2, lockstep=False)
    assert b[4] == {"sessions": 0, "cycles": 0, "steps": 0, "launches": 0}
    for u in range(2):
        for i in range(len(members)):
            for key in KEYS:
                assert a[2][u][i][key] == b[2][u][i][key]
    for x, y in zip(a[3], b[3]):
        assert np.array_equal(x, y)


@pytest.mark.parametrize("graph", [False, True])
def test_lockstep_member_failure_is_isolated(graph):
    """A member whose GMRES reaches its iteration limit fails alone; the other lockstep members
    complete the same update with their single-run rows."""
    from dg_hdg_euler_cpp_b200.solver import Batch, _lib

    members = [dict(COMMON, method="dg", precision="mixed", **DG_MEMBERS[0]),
               dict(COMMON, method="dg", precision="mixed", **dict(DG_MEMBERS[2], max_linear=3)),
               dict(COMMON, method="dg", precision="mixed", **DG_MEMBERS[1])]
    b = Batch(members)
    b.gmres_graph(graph)
    b.lockstep(True)
    u0 = start_states(b, members, AMPLITUDES[:3])
    b.stage_begin(u0)
    st = (_lib.dgh_update_stats * 3)()
    status = (ctypes.c_int * 3)()
    rc = b.lib.dgh_batch_newton_update(b.h, st, status)
    assert rc != 0 and list(status)[0] == 0 and list(status)[2] == 0 and list(status)[1] != 0
    assert "GMRES iteration limit reached" in b.lib.dgh_batch_error(b.h, 1).decode()
    finals = [b.state(0), b.state(2)]
    b.close()
    for j, i in enumerate((0, 2)):
        _, ref_rows, ref_state = single_run(members[i], u0[i], 1)
        assert st[i].krylov_iterations == ref_rows[0]["krylov_iterations"]
        assert st[i].residual_physical_rms == ref_rows[0]["residual_physical_rms"]
        assert np.array_equal(finals[j], ref_state)


def test_lockstep_group_validation():
    """dgh_lockstep_create refuses members it cannot advance together."""
    from dg_hdg_euler_cpp_b200.solver import Solver, _lib

    lib = _lib.load()
    a = Solver(**COMMON, method="dg", precision="mixed", nx=4, ny=4, k=2)
    b = Solver(**COMMON, method="dg", precision="fp64", nx=4, ny=4, k=3)
    c = Solver(**COMMON, method="dg", precision="mixed", nx=4, ny=4, k=2, quad=6)
    for pair, msg in (((a, b), "share one precision"), ((a, c), "collocated volume rule"), ((a, a), "listed twice")):
        arr = (ctypes.c_void_p * 2)(pair[0].h, pair[1].h)
        out = ctypes.c_void_p()
        assert lib.dgh_lockstep_create(arr, 2, ctypes.byref(out)) == 1
        assert msg in lib.dgh_lockstep_error().decode()
    for s in (a, b, c):
        s.close()
