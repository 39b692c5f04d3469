"""Python mirror of the reference's solver surface over the C ABI (include/dgh_gpu.h).

`Solver` exposes the calls of the reference's Problem (discretization.hpp:7-45), DGOperator
(dg_operator.hpp:5-17), BlockJacobi (block_jacobi.hpp:7-47), HybridOperator (hybrid.hpp:6-32)
and GMRES (gmres.hpp:21-35) with the same names and argument meaning, and `advance` mirrors
TimeIntegrator::advance (time_integrator.hpp:21-40).  Vectors are torch CUDA tensors (FP64) in
the reference layout; torch only provides device memory here, every kernel is the library's.
Errors raise DGHError carrying the reference's require() message.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib

METHODS = {"dg": 0, "hdg": 1, "both": 2}
INTEGRATORS = {"ssp-dirk3": 0, "be": 1}
TESTCASES = {"diagonal": 0, "wave": 1, "axis": 2}
PRECISIONS = {"fp64": 0, "mixed": 1, "mixed16": 2}
PRECONDITIONERS = {"block-jacobi": 0, "block-ilu0": 1}
OPS = {"dg": 0, "hdg": 1, "dg_t": 2}


class DGHError(RuntimeError):
    def __init__(self, code: int, message: str):
        super().__init__(message)
        self.code = code


def make_config(**kw) -> _lib.dgh_config:
    lib = _lib.load()
    cfg = _lib.dgh_config()
    lib.dgh_config_default(ctypes.byref(cfg))
    aliases = {"k": "degree", "ntol": "nonlinear_tolerance", "ltol": "linear_tolerance", "T": "final_time",
               "cells": "nx", "quad": "quadrature", "precond": "preconditioner"}
    for key, val in kw.items():
        key = aliases.get(key, key)
        if key == "method":
            val = METHODS[val] if isinstance(val, str) else val
        elif key == "integrator":
            val = INTEGRATORS[val] if isinstance(val, str) else val
        elif key == "testcase":
            val = TESTCASES[val] if isinstance(val, str) else val
        elif key == "precision":
            val = PRECISIONS[val] if isinstance(val, str) else val
        elif key == "preconditioner":
            val = PRECONDITIONERS[val] if isinstance(val, str) else val
        if not hasattr(cfg, key):
            raise KeyError(key)
        setattr(cfg, key, val)
    return cfg


def _ptr(t) -> ctypes.c_void_p:
    return ctypes.c_void_p(t.data_ptr())


class Solver:
    """One GPU context: the Problem plus the DG and/or HDG operators of one configuration.
    Solver(dim=1, cells=..., k=...) is the 1D problem of dg_hdg_1d (three variables per node,
    NVAR values per face trace).  Solver(comm=SlabComm, ...) is one rank's slab of the mesh
    (dgh_ctx_create_slab): its vectors carry a ghost cell row below and above the slab's rows;
    `slab` describes the slab and `interior(v)` is the view of a vector without its ghosts."""

    def __init__(self, comm: "SlabComm | None" = None, **kw):
        import torch

        self.torch = torch
        self.lib = _lib.load()
        self.cfg = make_config(**kw)
        h = ctypes.c_void_p()
        if comm is None:
            rc = self.lib.dgh_ctx_create(ctypes.byref(self.cfg), ctypes.byref(h))
        else:
            rc = self.lib.dgh_ctx_create_slab(ctypes.byref(self.cfg), comm.h, ctypes.byref(h))
        if rc != 0:
            raise DGHError(rc, self.lib.dgh_last_error(None).decode())
        self.h = h
        self.comm = comm  # the communicator outlives the context
        self.slab = None
        if comm is not None:
            info = (ctypes.c_int64 * 8)()
            self._rc(self.lib.dgh_slab_info(self.h, info))
            self.slab = dict(zip(("row0", "rows", "rank", "size", "offset", "length", "above", "face_row"),
                                 (int(x) for x in info)))
        s = (ctypes.c_int64 * 8)()
        self._rc(self.lib.dgh_sizes(self.h, s))
        self.size, self.trace_size, self.block, self.cells, self.faces, self.n, self.local_trace, self.face_width = (
            int(x) for x in s)
        g = (ctypes.c_double * 4)()
        self._rc(self.lib.dgh_geometry(self.h, g))
        self.hx, self.hy, self.lx, self.ly = list(g)
        self.dim = int(self.cfg.dim)
        self.nvar = 3 if self.dim == 1 else 4
        self.device = torch.device("cuda", self.cfg.device)

    def close(self):
        if getattr(self, "h", None):
            self.lib.dgh_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---- plumbing
    def _rc(self, rc: int):
        if rc != 0:
            raise DGHError(rc, self.lib.dgh_last_error(self.h).decode())

    def _call(self, name, *args):
        self.torch.cuda.synchronize(self.device)
        self._rc(getattr(self.lib, name)(self.h, *args))
        self._rc(self.lib.dgh_sync(self.h))

    def vec(self, n=None):
        return self.torch.zeros(self.size if n is None else n, dtype=self.torch.float64, device=self.device)

    def interior(self, v):
        """The slab's own rows of a volume vector (the whole vector outside a slab)."""
        if self.slab is None:
            return v
        return v[self.slab["offset"]:self.slab["offset"] + self.slab["length"]]

    def owned_faces(self, lam):
        """The slab's own faces of a trace vector (x faces, then upper y faces, of its rows),
        concatenated; the whole vector outside a slab."""
        if self.slab is None:
            return lam
        fr, rows, half = self.slab["face_row"], self.slab["rows"], self.trace_size // 2
        return self.torch.cat([lam[fr:fr * (rows + 1)], lam[half + fr:half + fr * (rows + 1)]])

    def tensor(self, a):
        return self.torch.as_tensor(np.ascontiguousarray(a, dtype=np.float64), device=self.device)

    def stream(self):
        return self.lib.dgh_stream(self.h)

    def launch_count(self) -> int:
        return int(self.lib.dgh_launch_count(self.h))

    def device_bytes(self) -> int:
        b = ctypes.c_int64()
        self._rc(self.lib.dgh_device_bytes(self.h, ctypes.byref(b)))
        return int(b.value)

    # ---- Problem
    def initial(self):
        u = self.vec()
        self._call("dgh_initial", _ptr(u))
        return u

    def freeze(self, u) -> float:
        r = ctypes.c_double()
        self._call("dgh_freeze", _ptr(u), ctypes.byref(r))
        return r.value

    def set_stage(self, old, step: float):
        self._call("dgh_set_stage", _ptr(old), ctypes.c_double(step))

    def residual(self, u):
        r = self.vec()
        self._call("dgh_residual", _ptr(u), _ptr(r))
        return r

    def admissible(self, u) -> bool:
        ok = ctypes.c_int()
        self._call("dgh_admissible", _ptr(u), ctypes.byref(ok))
        return bool(ok.value)

    def trace(self, u):
        lam = self.vec(self.trace_size)
        self._call("dgh_trace", _ptr(u), _ptr(lam))
        return lam

    def dual_norm(self, r) -> float:
        v = ctypes.c_double()
        self._call("dgh_dual_norm", _ptr(r), ctypes.byref(v))
        return v.value

    def state_norm(self, u) -> float:
        v = ctypes.c_double()
        self._call("dgh_state_norm", _ptr(u), ctypes.byref(v))
        return v.value

    def residual_rms(self, r) -> float:
        return self.dual_norm(r) / float(np.sqrt(self.lx * self.ly))

    def integral(self, u) -> np.ndarray:
        out = (ctypes.c_double * 4)()
        self._call("dgh_integral", _ptr(u), out)
        return np.array(out[:self.nvar])

    def l2_error(self, u, time: float) -> np.ndarray:
        out = (ctypes.c_double * 4)()
        self._call("dgh_l2_error", _ptr(u), ctypes.c_double(time), out)
        return np.array(out[:self.nvar])

    def speeds(self) -> np.ndarray:
        ab = np.zeros(2 * self.faces * (1 if self.dim == 1 else self.n))
        self._call("dgh_speeds", ab.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
        return ab.reshape(-1, 2)

    # ---- DGOperator
    def dg_refresh(self, u):
        self._call("dgh_dg_refresh", _ptr(u))

    def dg_apply(self, v):
        out = self.vec()
        self._call("dgh_dg_apply", _ptr(v), _ptr(out))
        return out

    def dg_apply_T(self, w):
        out = self.vec()
        self._call("dgh_dg_apply_T", _ptr(w), _ptr(out))
        return out

    def dg_block(self, row: int, col: int) -> np.ndarray:
        out = np.zeros(self.block * self.block)
        self._call("dgh_dg_block", row, col, out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
        return out.reshape(self.block, self.block)

    # ---- BlockJacobi
    def precond_refresh(self, op: str):
        self._call("dgh_block_jacobi_refresh", OPS[op])

    def precond_apply(self, op: str, x):
        z = self.vec(self.trace_size if op == "hdg" else self.size)
        self._call("dgh_precond_apply", OPS[op], _ptr(x), _ptr(z))
        return z

    # ---- HybridOperator
    def hdg_refresh_projected(self, u, r):
        self._call("dgh_hdg_refresh_projected", _ptr(u), _ptr(r))

    def hdg_rhs(self):
        out = self.vec(self.trace_size)
        self._call("dgh_hdg_rhs", _ptr(out))
        return out

    def hdg_apply(self, lam):
        out = self.vec(self.trace_size)
        self._call("dgh_hdg_apply", _ptr(lam), _ptr(out))
        return out

    def hdg_block(self, row: int, col: int) -> np.ndarray:
        fw = self.face_width
        out = np.zeros(fw * fw)
        self._call("dgh_hdg_block", row, col, out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
        return out.reshape(fw, fw)

    def hdg_recover(self, dlam):
        out = self.vec()
        self._call("dgh_hdg_recover", _ptr(dlam), _ptr(out))
        return out

    def hdg_retarget(self, r):
        """Retarget the FP32-condensed system to volume residual r (dgh_hdg_retarget)."""
        self._call("dgh_hdg_retarget", _ptr(r))

    def hdg_recovered_residual(self, e):
        out = self.vec()
        self._call("dgh_hdg_recovered_residual", _ptr(e), _ptr(out))
        return out

    def autotune_report(self) -> dict:
        """Factorisation variants and the DG block-solve grid shape in use, with the last tuning times
        (dgh_autotune_report, dgh_autotune_shapes)."""
        out = (ctypes.c_double * 6)()
        self._rc(self.lib.dgh_autotune_report(self.h, out))
        shape = (ctypes.c_double * 6)()
        self._rc(self.lib.dgh_autotune_shapes(self.h, shape))
        return {"dg_variant": int(out[0]), "hdg_variant": int(out[1]),
                "tune_ms": {"dg": [out[2], out[3]], "hdg": [out[4], out[5]]},
                "solve_shape": int(shape[0]), "solve_ms": [shape[1], shape[2]],
                "fused_ctas": int(shape[3]), "fused_ms": [shape[4], shape[5]]}

    def solve_shape(self, shape: int):
        """Grid shape of the DG block-Jacobi solves, 0 or 1 (dgh_shape_set)."""
        self._rc(self.lib.dgh_shape_set(self.h, 0, int(shape)))

    def fused_ctas(self, ctas: int):
        """CTAs per SM of the fused reduced-precision DG factorisation, 1 or 2 (dgh_shape_set)."""
        self._rc(self.lib.dgh_shape_set(self.h, 1, int(ctas)))

    # ---- GMRES
    def gmres_graph(self, on: bool = True):
        """Replay each GMRES restart cycle as one CUDA graph (dgh_gmres_graph_enable)."""
        self._rc(self.lib.dgh_gmres_graph_enable(self.h, 1 if on else 0))

    def gmres(self, op: str, rhs, limit: int, tol: float):
        """Returns (x, iterations, relative residual, true residual)."""
        x = self.vec(self.trace_size if op == "hdg" else self.size)
        it, rel = ctypes.c_int(), ctypes.c_double()
        self._call("dgh_gmres", OPS[op], _ptr(rhs), _ptr(x), limit, ctypes.c_double(tol), ctypes.byref(it),
                   ctypes.byref(rel))
        res_ptr = self.lib.dgh_gmres_residual(self.h, OPS[op])
        res = self.vec(x.numel())
        self._call("dgh_axpby", ctypes.c_double(1.0), ctypes.c_void_p(res_ptr), ctypes.c_double(0.0),
                   ctypes.c_void_p(res_ptr), _ptr(res), x.numel())
        return x, it.value, rel.value, res

    # ---- TimeIntegrator
    def advance(self, method: str, solution: np.ndarray, max_updates: int = 100000):
        """TimeIntegrator::advance on a host state; returns (state, run stats dict, update rows)."""
        it = ctypes.c_void_p()
        self._rc(self.lib.dgh_integrator_create(self.h, METHODS[method], ctypes.byref(it)))
        try:
            sol = np.ascontiguousarray(solution, dtype=np.float64).copy()
            st = _lib.dgh_run_stats()
            rows = (_lib.dgh_update_stats * max_updates)()
            rc = self.lib.dgh_advance(it, sol.ctypes.data_as(ctypes.c_void_p), ctypes.byref(st), rows, max_updates)
            if rc != 0:
                raise DGHError(rc, self.lib.dgh_integrator_error(it).decode())
            stats = {f: getattr(st, f) for f, _ in _lib.dgh_run_stats._fields_}
            ups = [{f: getattr(rows[i], f) for f, _ in _lib.dgh_update_stats._fields_}
                   for i in range(min(st.updates_recorded, max_updates))]
            return sol, stats, ups
        finally:
            self.lib.dgh_integrator_destroy(it)


class Integrator:
    """Single Newton updates of one backward-Euler stage (the speed protocol's unit of work)."""

    def __init__(self, solver: Solver, method: str):
        self.s = solver
        self.lib = solver.lib
        self.h = ctypes.c_void_p()
        solver._rc(self.lib.dgh_integrator_create(solver.h, METHODS[method], ctypes.byref(self.h)))

    def _rc(self, rc):
        if rc != 0:
            raise DGHError(rc, self.lib.dgh_integrator_error(self.h).decode())

    def stage_begin(self, u) -> float:
        dt = ctypes.c_double()
        self.s.torch.cuda.synchronize(self.s.device)
        self._rc(self.lib.dgh_stage_begin(self.h, _ptr(u), ctypes.byref(dt)))
        return dt.value

    def update(self) -> dict:
        st = _lib.dgh_update_stats()
        self._rc(self.lib.dgh_newton_update(self.h, ctypes.byref(st)))
        return {f: getattr(st, f) for f, _ in _lib.dgh_update_stats._fields_}

    def state_ptr(self) -> int:
        return int(self.lib.dgh_integrator_state(self.h))

    def set_limits(self, hdg_attempts: int = 4, line_search: int = 30):
        """Override the Schur attempts and Armijo halvings (dgh_integrator_set_limits)."""
        self._rc(self.lib.dgh_integrator_set_limits(self.h, hdg_attempts, line_search))

    def close(self):
        if self.h:
            self.lib.dgh_integrator_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class BlockJacobi:
    """A standalone pool of dense blocks factored on the device (BlockJacobi,
    block_jacobi.hpp:7-47): factor(blocks) with one of the LU kernels, apply(x) = A^{-1} x per
    block.  variant 0 left-looking FP64 tensor-pipe LU, 1 right-looking blocked LU, 2 one-warp LU
    (m <= 64), 3 FP64 LU with FP32 explicit inverses (m <= 64, mixed)."""

    def __init__(self, m: int, count: int, precision: str = "fp64", variant: int = 0, device: int = 0):
        import torch

        self.torch = torch
        self.lib = _lib.load()
        self.m, self.count = m, count
        self.device = torch.device("cuda", device)
        h = ctypes.c_void_p()
        rc = self.lib.dgh_block_jacobi_create(m, count, PRECISIONS[precision], variant, device, ctypes.byref(h))
        if rc != 0:
            raise DGHError(rc, self.lib.dgh_block_jacobi_error(None).decode())
        self.h = h

    def _rc(self, rc):
        if rc != 0:
            raise DGHError(rc, self.lib.dgh_block_jacobi_error(self.h).decode())

    def factor(self, blocks: np.ndarray):
        b = self.torch.as_tensor(np.ascontiguousarray(blocks, dtype=np.float64).reshape(-1), device=self.device)
        self.torch.cuda.synchronize(self.device)
        self._rc(self.lib.dgh_block_jacobi_factor(self.h, _ptr(b)))

    def apply(self, x: np.ndarray) -> np.ndarray:
        xt = self.torch.as_tensor(np.ascontiguousarray(x, dtype=np.float64), device=self.device)
        z = self.torch.zeros_like(xt)
        self.torch.cuda.synchronize(self.device)
        self._rc(self.lib.dgh_block_jacobi_apply(self.h, _ptr(xt), _ptr(z)))
        return z.cpu().numpy()

    def perm(self) -> np.ndarray:
        out = np.zeros(self.m * self.count, dtype=np.int32)
        self._rc(self.lib.dgh_block_jacobi_perm(self.h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_int))))
        return out.reshape(self.count, self.m)

    def close(self):
        if getattr(self, "h", None):
            self.lib.dgh_block_jacobi_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Batch:
    """Independent uneven member problems advanced together (dgh_batch_*): each member has its
    own config (mesh, degree, method "dg" or "hdg", precision ...), context, integrator and host
    thread, so the members' kernels overlap on the device; each member computes exactly what
    its single-problem run computes."""

    def __init__(self, members: list[dict]):
        self.lib = _lib.load()
        self.count = len(members)
        self.cfgs = (_lib.dgh_config * self.count)(*[make_config(**m) for m in members])
        h = ctypes.c_void_p()
        rc = self.lib.dgh_batch_create(self.cfgs, self.count, ctypes.byref(h))
        if rc != 0:
            raise DGHError(rc, self.lib.dgh_batch_error(None, 0).decode())
        self.h = h
        self.sizes = []
        for i in range(self.count):
            ctx = ctypes.c_void_p()
            self.lib.dgh_batch_member(self.h, i, ctypes.byref(ctx), None)
            s = (ctypes.c_int64 * 8)()
            self.lib.dgh_sizes(ctx, s)
            self.sizes.append(int(s[0]))

    def gmres_graph(self, on: bool = True):
        """Replay every member's GMRES restart cycles as CUDA graphs (dgh_gmres_graph_enable)."""
        for i in range(self.count):
            rc = self.lib.dgh_gmres_graph_enable(self.member_ctx(i), 1 if on else 0)
            if rc != 0:
                raise DGHError(rc, self.lib.dgh_last_error(self.member_ctx(i)).decode())

    def lockstep(self, on: bool = True):
        """Run the 2D DG members' GMRES solves in lockstep, each Arnoldi phase one launch over all
        members of a group (dgh_batch_lockstep)."""
        rc = self.lib.dgh_batch_lockstep(self.h, 1 if on else 0)
        if rc != 0:
            raise DGHError(rc, self.lib.dgh_batch_error(None, 0).decode())

    def lockstep_report(self) -> dict:
        """Sessions, restart cycles, Arnoldi steps and kernel launches of the lockstep groups."""
        out = (ctypes.c_int64 * 4)()
        rc = self.lib.dgh_batch_lockstep_report(self.h, out)
        if rc != 0:
            raise DGHError(rc, "dgh_batch_lockstep_report")
        return {"sessions": out[0], "cycles": out[1], "steps": out[2], "launches": out[3]}

    def _check(self, rc, status):
        if rc != 0:
            bad = [i for i in range(self.count) if status[i] != 0]
            msg = "; ".join(f"member {i}: {self.lib.dgh_batch_error(self.h, i).decode()}" for i in bad)
            raise DGHError(rc, msg)

    def member_ctx(self, i: int) -> ctypes.c_void_p:
        ctx = ctypes.c_void_p()
        self.lib.dgh_batch_member(self.h, i, ctypes.byref(ctx), None)
        return ctx

    def initial(self, i: int) -> np.ndarray:
        """Member i's projected initial state (dgh_initial), on the host."""
        ctx = self.member_ctx(i)
        out = np.empty(self.sizes[i])
        dev = ctypes.POINTER(ctypes.c_double)()
        self.lib.dgh_vec_alloc(ctx, self.sizes[i], ctypes.byref(dev))
        try:
            rc = self.lib.dgh_initial(ctx, dev)
            if rc == 0:
                rc = self.lib.dgh_download(ctx, out.ctypes.data_as(ctypes.c_void_p), dev, self.sizes[i])
            if rc != 0:
                raise DGHError(rc, self.lib.dgh_last_error(ctx).decode())
        finally:
            self.lib.dgh_vec_free(ctx, dev)
        return out

    def stage_begin(self, states=None) -> list[float]:
        """Every member starts a backward-Euler stage from states[i] (host arrays; None = its
        initial state); returns the members' step sizes."""
        keep = [None if states is None or states[i] is None else np.ascontiguousarray(states[i], dtype=np.float64)
                for i in range(self.count)]
        ptrs = (ctypes.c_void_p * self.count)(*[None if a is None else a.ctypes.data for a in keep])
        dt = (ctypes.c_double * self.count)()
        status = (ctypes.c_int * self.count)()
        rc = self.lib.dgh_batch_stage_begin(self.h, ptrs, dt, status)
        self._check(rc, status)
        return list(dt)

    def update(self) -> list[dict]:
        """One Newton update of every member; the members' rows."""
        st = (_lib.dgh_update_stats * self.count)()
        status = (ctypes.c_int * self.count)()
        rc = self.lib.dgh_batch_newton_update(self.h, st, status)
        self._check(rc, status)
        return [{f: getattr(s, f) for f, _ in _lib.dgh_update_stats._fields_} for s in st]

    def state(self, i: int) -> np.ndarray:
        out = np.empty(self.sizes[i])
        rc = self.lib.dgh_batch_download(self.h, i, out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
        if rc != 0:
            raise DGHError(rc, self.lib.dgh_batch_error(self.h, i).decode())
        return out

    def close(self):
        if getattr(self, "h", None):
            self.lib.dgh_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---- slab domain decomposition ------------------------------------------------------------------
def slab_rows(ny: int, size: int, rank: int) -> tuple[int, int, int, int]:
    """(first global row, rows, rank below, rank above) of rank `rank` (dgh_slab_rows)."""
    lib = _lib.load()
    out = (ctypes.c_int * 4)()
    rc = lib.dgh_slab_rows(ny, size, rank, out)
    if rc != 0:
        raise DGHError(rc, f"no slab partition of {ny} rows over {size} ranks for rank {rank}")
    return tuple(int(x) for x in out)


class SlabComm:
    """One rank's communicator of the slab decomposition (dgh_comm_*): NCCL across processes and
    GPUs, or an in-process group whose ranks are host threads (several slabs on one GPU)."""

    def __init__(self, handle: ctypes.c_void_p):
        self.lib = _lib.load()
        self.h = handle
        info = (ctypes.c_int * 3)()
        self.lib.dgh_comm_info(self.h, info)
        self.rank, self.size = int(info[0]), int(info[1])
        self.kind = "nccl" if info[2] == 1 else "local"

    @staticmethod
    def _check(rc: int):
        if rc != 0:
            raise DGHError(rc, _lib.load().dgh_comm_error().decode())

    @classmethod
    def local_group(cls, size: int, timeout_ms: int = 60000) -> list["SlabComm"]:
        lib = _lib.load()
        hs = (ctypes.c_void_p * size)()
        cls._check(lib.dgh_comm_local_create(size, timeout_ms, hs))
        return [cls(ctypes.c_void_p(h)) for h in hs]

    @staticmethod
    def nccl_unique_id() -> bytes:
        buf = (ctypes.c_ubyte * 128)()
        SlabComm._check(_lib.load().dgh_comm_nccl_unique_id(buf))
        return bytes(buf)

    @classmethod
    def nccl(cls, unique_id: bytes, size: int, rank: int, device: int) -> "SlabComm":
        buf = (ctypes.c_ubyte * 128).from_buffer_copy(unique_id)
        h = ctypes.c_void_p()
        cls._check(_lib.load().dgh_comm_nccl_create(buf, size, rank, device, ctypes.byref(h)))
        return cls(h)

    def fail(self, why: str = "failed by its host"):
        self.lib.dgh_comm_fail(self.h, why.encode())

    def set_timeout(self, timeout_ms: int):
        """How long this rank waits for its peers (dgh_comm_set_timeout)."""
        self._check(self.lib.dgh_comm_set_timeout(self.h, timeout_ms))

    def close(self):
        if self.h:
            self.lib.dgh_comm_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def share_unique_id(make_id=None, group=None) -> bytes:
    """Rank 0's NCCL id, broadcast to every rank of the initialised torch.distributed group (any
    backend)."""
    import torch.distributed as dist

    box = [(make_id or SlabComm.nccl_unique_id)() if dist.get_rank(group) == 0 else None]
    dist.broadcast_object_list(box, src=0, group=group)
    return box[0]


def nccl_slab_comm(device: int, group=None) -> SlabComm:
    """This process's NCCL slab communicator over the torch.distributed group (one rank per GPU)."""
    import torch.distributed as dist

    uid = share_unique_id(group=group)
    return SlabComm.nccl(uid, dist.get_world_size(group), dist.get_rank(group), device)


def run_ranks(comms: list[SlabComm], body) -> list:
    """Runs body(rank, comm) for every rank of an in-process group, each on its own host thread;
    returns the results in rank order.  A rank that raises fails the group (its peers then leave
    their collectives with DGH_ERR_COMM instead of waiting), and the first error is re-raised."""
    import threading

    results, errors = [None] * len(comms), [None] * len(comms)

    def run(r):
        try:
            results[r] = body(r, comms[r])
        except BaseException as e:  # noqa: BLE001 — reported below, after every rank has ended
            errors[r] = e
            comms[r].fail(f"{type(e).__name__}: {e}")

    threads = [threading.Thread(target=run, args=(r,)) for r in range(len(comms))]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    for e in errors:
        if e is not None:
            raise e
    return results


# ---- the uneven-batch workload: 16 members drawn from seeds 0-15 --------------------------------
_MASK64 = (1 << 64) - 1


def splitmix64(state: int) -> tuple[int, int]:
    """One step of Vigna's SplitMix64 generator: (output, next state)."""
    state = (state + 0x9E3779B97F4A7C15) & _MASK64
    z = state
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & _MASK64
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & _MASK64
    return z ^ (z >> 31), state


def batch_member(seed: int, sizes=(32, 64, 96, 128), degrees=(2, 4, 6, 8), precision="mixed") -> dict:
    """Member `seed` of the uneven batch: degree k, an N x N mesh, amplitude A in [0.05, 0.25)
    and the method, drawn from SplitMix64 seeded by the seed index; backward Euler at CFL 5 with
    GMRES(30)."""
    st = seed
    r = []
    for _ in range(4):
        v, st = splitmix64(st)
        r.append(v)
    k = degrees[r[0] % len(degrees)]
    n = sizes[r[1] % len(sizes)]
    amp = 0.05 + 0.2 * ((r[2] >> 11) / float(1 << 53))
    method = ("dg", "hdg")[r[3] % 2]
    return {"config": dict(nx=n, ny=n, k=k, cfl=5.0, integrator="be", steps=1, restart=30, max_linear=1500,
                           method=method, precision=precision),
            "amplitude": amp, "seed": seed}


def perturb(u: np.ndarray, nx: int, ny: int, k: int, amplitude: float) -> np.ndarray:
    """The member's initial state with every conserved variable scaled by
    1 + A sin(2 pi X) sin(2 pi Y), X and Y the mesh-relative node coordinates (periodic, and
    positive density and pressure for A < 1)."""
    n = k + 1
    xi, _ = np.polynomial.legendre.leggauss(n)
    s = (xi + 1) / 2
    X = (np.arange(nx)[:, None] + s[None, :]) / nx   # [cx][i]
    Y = (np.arange(ny)[:, None] + s[None, :]) / ny   # [cy][j]
    f = 1 + amplitude * np.sin(2 * np.pi * Y)[:, None, :, None] * np.sin(2 * np.pi * X)[None, :, None, :]
    # f[cy][cx][j][i] -> per cell (cell = cy * nx + cx), per node (j, i), same for all 4 variables
    f = f.reshape(ny * nx, 1, n, n)
    return (u.reshape(ny * nx, 4, n, n) * f).reshape(-1)
