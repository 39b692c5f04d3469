"""Batched uneven problems (dgh_batch_*): members with different meshes, degrees, methods and
precisions advanced together equal their single-problem runs bitwise (update rows and states),
and a failing member reports its own error while the others complete."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MEMBERS = [
    dict(nx=6, ny=6, k=2, method="dg", precision="fp64"),
    dict(nx=8, ny=5, k=3, method="hdg", precision="mixed"),
    dict(nx=4, ny=4, k=5, method="dg", precision="mixed"),
    dict(nx=5, ny=7, k=4, method="hdg", precision="fp64"),
    dict(dim=1, cells=24, k=3, method="hdg"),
    dict(dim=1, cells=40, k=2, method="dg"),
]
COMMON = dict(cfl=5.0, integrator="be", steps=1, restart=30, max_linear=1500)
AMPLITUDES = [0.1, 0.2, 0.05, 0.15, 0.0, 0.0]


def states_for(batch):
    from dg_hdg_euler_cpp_b200.solver import perturb

    out = []
    for i, (m, a) in enumerate(zip(MEMBERS, AMPLITUDES)):
        u = batch.initial(i)
        out.append(perturb(u, m["nx"], m["ny"], m["k"], a) if m.get("dim", 2) == 2 else u)
    return out


def single_run(kw, u0, updates):
    import ctypes

    from dg_hdg_euler_cpp_b200.solver import Integrator, Solver

    s = Solver(**COMMON, **kw)
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


KEYS = ("krylov_iterations", "residual_physical_rms", "linear_relative_residual", "dg_linear_relative_residual",
        "damping", "dt", "cfl")


@pytest.mark.parametrize("graph", [False, True])
def test_batch_members_equal_single_runs_bitwise(graph):
    """Single runs launch their GMRES cycles step by step; the batch either way."""
    from dg_hdg_euler_cpp_b200.solver import Batch

    b = Batch([dict(COMMON, **m) for m in MEMBERS])
    b.gmres_graph(graph)
    u0 = states_for(b)
    dts = b.stage_begin(u0)
    rows = [b.update() for _ in range(3)]
    finals = [b.state(i) for i in range(b.count)]
    b.close()
    for i, kw in enumerate(MEMBERS):
        dt, ref_rows, ref_state = single_run(kw, u0[i], 3)
        assert dts[i] == dt, i
        for u in range(3):
            for key in KEYS:
                assert rows[u][i][key] == ref_rows[u][key], (i, u, key)
        assert np.array_equal(finals[i], ref_state), i


def test_batch_default_initial_states_and_restart_of_stage():
    """NULL host states start from each member's dgh_initial state; a second stage_begin
    restarts the members exactly as the first did."""
    from dg_hdg_euler_cpp_b200.solver import Batch

    b = Batch([dict(COMMON, **m) for m in MEMBERS[:3]])
    dts = b.stage_begin()
    first = b.update()
    dts2 = b.stage_begin([b.initial(i) for i in range(b.count)])
    second = b.update()
    assert dts == dts2
    for a, c in zip(first, second):
        assert a["krylov_iterations"] == c["krylov_iterations"]
        assert a["residual_physical_rms"] == c["residual_physical_rms"]
    b.close()


def test_batch_member_failure_is_reported_per_member():
    from dg_hdg_euler_cpp_b200.solver import Batch, DGHError

    members = [dict(COMMON, **MEMBERS[0]), dict(COMMON, **dict(MEMBERS[2], max_linear=3))]
    b = Batch(members)
    b.stage_begin()
    with pytest.raises(DGHError, match=r"member 1: GMRES iteration limit reached") as e:
        b.update()
    assert "member 0" not in str(e.value)
    # the healthy member completed its update and can continue
    assert np.isfinite(b.state(0)).all()
    b.close()
