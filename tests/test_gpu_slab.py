"""Slab domain decomposition of the 2D DG Newton update (dgh_ctx_create_slab) on one GPU: the
mesh split into 1-3 slabs of cell rows, each slab its own context on its own host thread, the
ranks exchanging ghost rows and reduced scalars through an in-process group (host barriers
after stream synchronisation, so no kernel waits on another rank's kernel).  Checked against
the whole-mesh context: the interior of every slab's initial state, frozen rate, residual and
J*v bitwise; norms, integrals and L2 errors to rounding; backward-Euler Newton updates and
DIRK3 steps to the Krylov tolerance with the same dt.  Ghost rows of the inputs are NaN, so the
library's halo exchange must overwrite them.  An NCCL communicator of one rank must give the
in-process group's single-rank results bitwise.  A rank that fails on the host releases its
peers with DGH_ERR_COMM (no device fault involved)."""
import ctypes
import threading

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MESH = dict(nx=10, ny=9, k=3)
KEYS = ("krylov_iterations", "residual_physical_rms", "linear_relative_residual", "dg_linear_relative_residual",
        "damping", "dt", "cfl")  # the update statistics without the wall-clock field


def rows_of(v: np.ndarray, nx: int, m: int, row0: int, rows: int) -> np.ndarray:
    """Global rows [row0, row0 + rows) of a whole-mesh volume vector."""
    return v.reshape(-1, nx * m)[row0:row0 + rows].reshape(-1)


def to_slab(s, v_global: np.ndarray):
    """The slab's vector of a whole-mesh vector: its rows, NaN ghost rows."""
    nx, m = s.cfg.nx, s.block
    out = s.vec()
    out.fill_(float("nan"))
    s.interior(out).copy_(s.tensor(rows_of(v_global, nx, m, s.slab["row0"], s.slab["rows"])))
    return out


def gather(parts: list[np.ndarray]) -> np.ndarray:
    return np.concatenate(parts)


def whole(**kw):
    from dg_hdg_euler_cpp_b200.solver import Solver

    return Solver(**kw)


def run_slabs(size: int, body, timeout_ms: int = 60000):
    from dg_hdg_euler_cpp_b200.solver import SlabComm, run_ranks

    comms = SlabComm.local_group(size, timeout_ms)
    try:
        return run_ranks(comms, body)
    finally:
        for c in comms:
            c.close()


@pytest.mark.parametrize("size", [1, 2, 3])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_slab_operators_equal_whole_mesh(size, precision):
    from dg_hdg_euler_cpp_b200.solver import Solver, perturb

    kw = dict(MESH, cfl=5.0, integrator="be", steps=1, method="dg", precision=precision)
    nx, ny, k = MESH["nx"], MESH["ny"], MESH["k"]
    ref = whole(**kw)
    u0 = ref.initial()
    u = ref.tensor(perturb(u0.cpu().numpy(), nx, ny, k, 0.1))
    rate = ref.freeze(u)
    dt = 5.0 / rate
    ref.set_stage(u, dt)
    v = ref.tensor(np.sin(0.37 * np.arange(ref.size)))
    up = u + 1e-3 * v
    r = ref.residual(up).cpu().numpy()
    ref.dg_refresh(up)
    jv = ref.dg_apply(v).cpu().numpy()
    want = dict(u0=u0.cpu().numpy(), r=r, jv=jv, norm=ref.dual_norm(ref.tensor(r)), snorm=ref.state_norm(up),
                integral=ref.integral(up), l2=ref.l2_error(u0, 0.0))
    ref.close()

    def body(rank, comm):
        s = Solver(comm=comm, **kw)
        got = {"row0": s.slab["row0"], "rows": s.slab["rows"]}
        got["u0"] = s.interior(s.initial()).cpu().numpy()
        ul = to_slab(s, u.cpu().numpy())
        got["rate"] = s.freeze(ul)
        s.set_stage(ul, dt)
        upl = to_slab(s, up.cpu().numpy())
        rl = s.residual(upl)
        got["r_ghosts_zero"] = bool((rl[:s.slab["offset"]] == 0).all() and (rl[s.slab["offset"] + s.slab["length"]:] == 0).all())
        got["r"] = s.interior(rl).cpu().numpy()
        got["norm"] = s.dual_norm(rl)
        got["snorm"] = s.state_norm(to_slab(s, up.cpu().numpy()))
        got["integral"] = s.integral(to_slab(s, up.cpu().numpy()))
        got["l2"] = s.l2_error(to_slab(s, u0.cpu().numpy()), 0.0)
        s.dg_refresh(to_slab(s, up.cpu().numpy()))
        got["jv"] = s.interior(s.dg_apply(to_slab(s, v.cpu().numpy()))).cpu().numpy()
        s.close()
        return got

    ranks = run_slabs(size, body)
    assert sum(g["rows"] for g in ranks) == ny
    m = 4 * (k + 1) ** 2
    for g in ranks:
        assert g["rate"] == rate  # a maximum: the same bits on every rank
        assert g["r_ghosts_zero"]
        for key in ("u0", "r", "jv"):
            assert np.array_equal(g[key], rows_of(want[key], nx, m, g["row0"], g["rows"])), (key, g["row0"])
        assert abs(g["norm"] - want["norm"]) <= 1e-13 * want["norm"]
        assert abs(g["snorm"] - want["snorm"]) <= 1e-13 * want["snorm"]
        assert np.allclose(g["integral"], want["integral"], rtol=1e-13, atol=1e-15)
        assert np.allclose(g["l2"], want["l2"], rtol=1e-12, atol=1e-18)
    # every rank received the same reduced scalars
    assert len({g["norm"] for g in ranks}) == 1 and len({g["snorm"] for g in ranks}) == 1


def newton_rows(kw, u_global, updates, comm=None):
    from dg_hdg_euler_cpp_b200.solver import Integrator, Solver

    s = Solver(comm=comm, **kw)
    it = Integrator(s, kw["method"])
    u = to_slab(s, u_global) if comm is not None else s.tensor(u_global)
    dt = it.stage_begin(u)
    rows = [it.update() for _ in range(updates)]
    state = s.vec()
    p = ctypes.c_void_p(it.state_ptr())
    s._rc(s.lib.dgh_axpby(s.h, 1.0, p, 0.0, p, ctypes.c_void_p(state.data_ptr()), state.numel()))
    s._rc(s.lib.dgh_sync(s.h))
    out = s.interior(state).cpu().numpy()
    it.close()
    s.close()
    return dt, rows, out


@pytest.mark.parametrize("size", [2, 3])
@pytest.mark.parametrize("precision", ["fp64", "mixed", "mixed16"])
def test_slab_newton_updates_match_whole_mesh(size, precision):
    """Backward Euler at CFL 5, GMRES(20): three Newton updates; dt bitwise, Krylov counts within
    one, residual rms and the state to the linear tolerance's reach."""
    from dg_hdg_euler_cpp_b200.solver import perturb

    kw = dict(nx=12, ny=12, k=3, cfl=5.0, integrator="be", steps=1, method="dg", precision=precision, restart=20)
    s0 = whole(**kw)
    u0 = perturb(s0.initial().cpu().numpy(), 12, 12, 3, 0.15)
    s0.close()
    dt, rows, state = newton_rows(kw, u0, 3)
    ranks = run_slabs(size, lambda rank, comm: newton_rows(kw, u0, 3, comm))
    got = gather([x[2] for x in ranks])
    scale = np.max(np.abs(state))
    for rdt, rrows, _ in ranks:
        assert rdt == dt
        for a, b in zip(rrows, rows):
            assert abs(a["krylov_iterations"] - b["krylov_iterations"]) <= 1, (a, b)
            assert abs(a["residual_physical_rms"] - b["residual_physical_rms"]) <= 1e-9 * rows[0]["residual_physical_rms"]
            assert a["damping"] == b["damping"]
    for a, b in zip(ranks[0][1], ranks[-1][1]):  # every rank reports the same statistics
        assert all(a[key] == b[key] for key in KEYS)
    assert np.max(np.abs(got - state)) <= 1e-10 * scale


def owned_of(lam: np.ndarray, nx: int, fw: int, cells: int, row0: int, rows: int) -> np.ndarray:
    """The faces of global rows [row0, row0 + rows) of a whole-mesh trace vector: x faces, then
    upper y faces."""
    fr, half = nx * fw, cells * fw
    return np.concatenate([lam[row0 * fr:(row0 + rows) * fr], lam[half + row0 * fr:half + (row0 + rows) * fr]])


def to_slab_trace(s, lam_global: np.ndarray, cells: int):
    """The slab's trace vector of a whole-mesh one: its own faces, NaN elsewhere."""
    fr, rows, row0 = s.slab["face_row"], s.slab["rows"], s.slab["row0"]
    out = s.vec(s.trace_size)
    out.fill_(float("nan"))
    half, ghalf = s.trace_size // 2, cells * s.face_width
    out[fr:fr * (rows + 1)] = s.tensor(lam_global[row0 * fr:(row0 + rows) * fr])
    out[half + fr:half + fr * (rows + 1)] = s.tensor(lam_global[ghalf + row0 * fr:ghalf + (row0 + rows) * fr])
    return out


@pytest.mark.parametrize("size", [1, 2, 3])
@pytest.mark.parametrize("precision,condense32", [("fp64", 0), ("mixed", 0), ("mixed", 1)])
def test_slab_hdg_operators_equal_whole_mesh(size, precision, condense32):
    """The condensed right-hand side, the Schur apply and the face traces of the state on owned
    faces, the recovery and the recovered residual on interior cells, bitwise; the trace inputs
    are NaN off the owned faces."""
    from dg_hdg_euler_cpp_b200.solver import Solver, perturb

    kw = dict(MESH, cfl=5.0, integrator="be", steps=1, method="hdg", precision=precision, condense32=condense32)
    nx, ny, k = MESH["nx"], MESH["ny"], MESH["k"]
    ref = whole(**kw)
    u = perturb(ref.initial().cpu().numpy(), nx, ny, k, 0.1)
    ut = ref.tensor(u)
    dt = 5.0 / ref.freeze(ut)
    ref.set_stage(ut, dt)
    r = ref.residual(ut)
    ref.hdg_refresh_projected(ut, r)
    lam = np.cos(0.29 * np.arange(ref.trace_size)) * 1e-3
    want = dict(rhs=ref.hdg_rhs().cpu().numpy(), sa=ref.hdg_apply(ref.tensor(lam)).cpu().numpy(),
                tr=ref.trace(ut).cpu().numpy(),
                du=ref.hdg_recover(ref.tensor(lam)).cpu().numpy(),
                rr=ref.hdg_recovered_residual(ref.tensor(lam)).cpu().numpy())
    cells, fw, m = ref.cells, ref.face_width, ref.block
    ref.close()

    def body(rank, comm):
        s = Solver(comm=comm, **kw)
        got = {"row0": s.slab["row0"], "rows": s.slab["rows"], "above": s.slab["above"]}
        ul = to_slab(s, u)
        s.freeze(ul)
        s.set_stage(ul, dt)
        rl = s.residual(ul)
        s.hdg_refresh_projected(ul, rl)
        got["rhs"] = s.owned_faces(s.hdg_rhs()).cpu().numpy()
        got["tr"] = s.owned_faces(s.trace(to_slab(s, u))).cpu().numpy()
        got["sa"] = s.owned_faces(s.hdg_apply(to_slab_trace(s, lam, cells))).cpu().numpy()
        got["du"] = s.interior(s.hdg_recover(to_slab_trace(s, lam, cells))).cpu().numpy()
        got["rr"] = s.interior(s.hdg_recovered_residual(to_slab_trace(s, lam, cells))).cpu().numpy()
        s.close()
        return got

    for g in run_slabs(size, body):
        assert g["above"] == 2
        for key in ("rhs", "sa", "tr"):
            assert np.array_equal(g[key], owned_of(want[key], nx, fw, cells, g["row0"], g["rows"])), (key, g["row0"])
        for key in ("du", "rr"):
            assert np.array_equal(g[key], rows_of(want[key], nx, m, g["row0"], g["rows"])), (key, g["row0"])


@pytest.mark.parametrize("size", [2, 3])
@pytest.mark.parametrize("precision,condense32", [("fp64", 0), ("mixed", 0), ("mixed", 1)])
def test_slab_hdg_newton_updates_match_whole_mesh(size, precision, condense32):
    """The condensed HDG Newton update on 2-3 slabs: three updates as in the DG test."""
    from dg_hdg_euler_cpp_b200.solver import perturb

    kw = dict(nx=12, ny=12, k=3, cfl=5.0, integrator="be", steps=1, method="hdg", precision=precision,
              condense32=condense32, restart=20)
    s0 = whole(**kw)
    u0 = perturb(s0.initial().cpu().numpy(), 12, 12, 3, 0.15)
    s0.close()
    dt, rows, state = newton_rows(kw, u0, 3)
    ranks = run_slabs(size, lambda rank, comm: newton_rows(kw, u0, 3, comm))
    got = gather([x[2] for x in ranks])
    for rdt, rrows, _ in ranks:
        assert rdt == dt
        for a, b in zip(rrows, rows):
            assert abs(a["krylov_iterations"] - b["krylov_iterations"]) <= 2, (a, b)
            assert abs(a["residual_physical_rms"] - b["residual_physical_rms"]) <= 1e-9 * rows[0]["residual_physical_rms"]
            assert a["damping"] == b["damping"]
    for a, b in zip(ranks[0][1], ranks[-1][1]):
        assert all(a[key] == b[key] for key in KEYS)
    assert np.max(np.abs(got - state)) <= 1e-10 * np.max(np.abs(state))


def test_slab_dirk3_advance_matches_whole_mesh():
    """dgh_advance on slab contexts: two DIRK3 steps (CFL 2) of the accuracy configuration's
    problem on an 8 x 8 mesh, k = 2; final interior states and run statistics."""
    kw = dict(nx=8, ny=8, k=2, cfl=2.0, integrator="ssp-dirk3", steps=2, method="dg", testcase="wave")
    s0 = whole(**kw)
    u0 = s0.initial().cpu().numpy()
    sol, stats, _ = s0.advance("dg", u0)
    s0.close()

    def body(rank, comm):
        from dg_hdg_euler_cpp_b200.solver import Solver

        s = Solver(comm=comm, **kw)
        host = to_slab(s, u0).cpu().numpy()
        out, st, _ = s.advance("dg", host)
        o, n = s.slab["offset"], s.slab["length"]
        s.close()
        return out[o:o + n], st

    ranks = run_slabs(2, body)
    got = gather([x[0] for x in ranks])
    assert np.max(np.abs(got - sol)) <= 1e-10 * np.max(np.abs(sol))
    for _, st in ranks:
        # the second step's dt comes from a state equal to rounding, so its rate may differ in the last bit
        assert st["steps"] == stats["steps"]
        assert abs(st["final_time"] - stats["final_time"]) <= 1e-14 * stats["final_time"]
        assert st["newton_iterations"] == stats["newton_iterations"]
        assert abs(st["conservation_drift"] - stats["conservation_drift"]) <= 1e-13


def test_nccl_single_rank_equals_local_single_rank():
    """The NCCL communicator (one rank, this GPU) against the in-process group of one rank."""
    from dg_hdg_euler_cpp_b200.solver import SlabComm, perturb

    kw = dict(nx=8, ny=7, k=4, cfl=5.0, integrator="be", steps=1, method="dg", precision="mixed", restart=20)
    s0 = whole(**kw)
    u0 = perturb(s0.initial().cpu().numpy(), 8, 7, 4, 0.1)
    s0.close()
    nccl = SlabComm.nccl(SlabComm.nccl_unique_id(), 1, 0, 0)
    assert nccl.kind == "nccl"
    a = newton_rows(kw, u0, 2, nccl)
    nccl.close()
    b = run_slabs(1, lambda rank, comm: newton_rows(kw, u0, 2, comm))[0]
    assert a[0] == b[0] and np.array_equal(a[2], b[2])
    for x, y in zip(a[1], b[1]):
        assert all(x[key] == y[key] for key in KEYS)


def test_rank_failure_releases_peers():
    """Rank 1 fails on the host before its first collective (fail), or never enters it (the
    group's timeout); rank 0, waiting in the halo exchange of its initial state, leaves with
    DGH_ERR_COMM either way."""
    from dg_hdg_euler_cpp_b200.solver import DGHError, SlabComm, Solver

    kw = dict(nx=6, ny=6, k=2, method="dg")
    for mode in ("fail", "absent"):
        comms = SlabComm.local_group(2, 1500)
        solvers = [Solver(comm=c, **kw) for c in comms]
        caught = {}

        def rank0():
            try:
                solvers[0].initial()
            except DGHError as e:
                caught["code"], caught["msg"] = e.code, str(e)

        t = threading.Thread(target=rank0)
        t.start()
        if mode == "fail":
            comms[1].fail("rank 1 raised before its update")
        t.join(timeout=60)
        assert not t.is_alive()
        assert caught.get("code") == 9, caught
        assert ("rank 1 raised" in caught["msg"]) if mode == "fail" else ("did not enter" in caught["msg"])
        for s in solvers:
            s.close()
        for c in comms:
            c.close()


def test_slab_refuses_graphs_and_lockstep():
    from dg_hdg_euler_cpp_b200 import _lib
    from dg_hdg_euler_cpp_b200.solver import DGHError, SlabComm, Solver

    comms = SlabComm.local_group(1)
    s = Solver(comm=comms[0], nx=6, ny=6, k=2, method="dg")
    with pytest.raises(DGHError, match="step by step"):
        s.gmres_graph(True)
    lib = _lib.load()
    arr = (ctypes.c_void_p * 1)(s.h)
    assert lib.dgh_lockstep_create(arr, 1, ctypes.byref(ctypes.c_void_p())) == 1
    assert "slab contexts" in lib.dgh_lockstep_error().decode()
    s.close()
    comms[0].close()


TWO_GPU_WORKER = r"""
import datetime, json, os, sys
sys.path.insert(0, sys.argv[1])
import numpy as np
import torch
import torch.distributed as dist
from dg_hdg_euler_cpp_b200.solver import Integrator, Solver, nccl_slab_comm, perturb
rank = int(os.environ["RANK"])
torch.cuda.set_device(rank)
dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=120))  # host plumbing: the NCCL id
comm = nccl_slab_comm(rank)
method = sys.argv[2]
kw = dict(nx=12, ny=12, k=3, cfl=5.0, integrator="be", steps=1, method=method, precision="mixed", restart=20,
          device=rank)
whole = Solver(**kw)
u0 = perturb(whole.initial().cpu().numpy(), 12, 12, 3, 0.15)
whole.close()


def run(s, u):
    it = Integrator(s, method)
    dt = it.stage_begin(u)
    rows = [it.update()["krylov_iterations"] for _ in range(2)]
    out = np.empty(s.size)
    import ctypes
    s.lib.dgh_download(s.h, out.ctypes.data_as(ctypes.c_void_p), ctypes.c_void_p(it.state_ptr()), s.size)
    it.close()
    return dt, rows, out


s = Solver(comm=comm, **kw)
m, row0, rows = s.block, s.slab["row0"], s.slab["rows"]
u = s.vec()
s.interior(u).copy_(s.tensor(u0.reshape(-1, 12 * m)[row0:row0 + rows].reshape(-1)))
dt, kry, out = run(s, u)
mine = out[s.slab["offset"]:s.slab["offset"] + s.slab["length"]]
s.close()
parts = [None, None]
dist.all_gather_object(parts, (dt, kry, mine.tolist()))
if rank == 0:
    ref = Solver(**kw)
    rdt, rkry, rout = run(ref, ref.tensor(u0))
    ref.close()
    got = np.concatenate([np.array(p[2]) for p in parts])
    print(json.dumps({"dt_equal": all(p[0] == rdt for p in parts), "krylov": [p[1] for p in parts],
                      "krylov_whole": rkry, "rel": float(np.max(np.abs(got - rout)) / np.max(np.abs(rout)))}))
comm.close()
dist.destroy_process_group()
"""


@pytest.mark.parametrize("method", ["dg", "hdg"])
def test_nccl_two_gpus_match_whole_mesh(method):
    """Two processes on two GPUs, one NCCL slab each (skipped with fewer GPUs): two Newton
    updates against the whole mesh on rank 0's GPU."""
    import json
    import os
    import subprocess
    import sys

    import torch

    from conftest import ROOT
    from test_dist_replicas import free_port

    if torch.cuda.device_count() < 2:
        pytest.skip("needs two GPUs")
    port = free_port()
    procs = []
    for rank in range(2):
        env = dict(os.environ, RANK=str(rank), WORLD_SIZE="2", MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
        procs.append(subprocess.Popen([sys.executable, "-c", TWO_GPU_WORKER, str(ROOT), method], env=env,
                                      stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True))
    outs = []
    for p in procs:
        out, err = p.communicate(timeout=600)
        assert p.returncode == 0, err[-2000:]
        outs.append(out)
    res = json.loads(outs[0].strip().splitlines()[-1])
    assert res["dt_equal"] and res["krylov"][0] == res["krylov"][1]
    assert all(abs(a - b) <= 1 for a, b in zip(res["krylov"][0], res["krylov_whole"]))
    assert res["rel"] <= 1e-10
