"""Test infrastructure only: ctypes wrapper over the CPU oracle (oracle/_bin/liboracle.so).

The oracle is a plain C++ restatement of the reference solver YueWu2002/DG_HDG_Euler_Cpp
(dg_hdg_2d/src, dg_hdg_1d/src, common/).  Only tests/, __graft_entry__.smoke() and bench.py's CPU
baseline use this module: to check the device results, and (the CPU baseline) as the timed CPU
restatement of the reference.  The product never loads it.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "_bin" / "liboracle.so"
CLI_PATH = HERE / "_bin" / "dgh2d_oracle"
CLI1D_PATH = HERE / "_bin" / "dgh1d_oracle"

_D = ctypes.POINTER(ctypes.c_double)
_lib = None


def build() -> None:
    """Compile the oracle with its Makefile (g++ only; no GPU needed)."""
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            build()
        _lib = ctypes.CDLL(str(LIB_PATH))
        _lib.oracle_create.restype = ctypes.c_void_p
        _lib.oracle_create.argtypes = [ctypes.c_char_p]
        _lib.oracle_error.restype = ctypes.c_char_p
        _lib.oracle_destroy.argtypes = [ctypes.c_void_p]
        _lib.oracle1d_create.restype = ctypes.c_void_p
        _lib.oracle1d_create.argtypes = [ctypes.c_char_p]
        _lib.oracle1d_destroy.argtypes = [ctypes.c_void_p]
    return _lib


def _p(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(_D)


class OracleError(RuntimeError):
    pass


class Oracle:
    """One oracle Problem plus its DG and HDG operators (dg_hdg_2d/include/euler/*.hpp)."""

    def __init__(self, args: str, threads: int | None = None):
        L = lib()
        L.oracle_set_threads(ctypes.c_int(threads or int(os.environ.get("DGH_ORACLE_THREADS", "1"))))
        self.h = L.oracle_create(args.encode())
        if not self.h:
            raise OracleError(L.oracle_error().decode())
        s = (ctypes.c_longlong * 6)()
        L.oracle_sizes(ctypes.c_void_p(self.h), s)
        self.size, self.trace_size, self.block, self.cells, self.faces, self.n = (int(x) for x in s)
        g = (ctypes.c_double * 4)()
        L.oracle_geometry(ctypes.c_void_p(self.h), g)
        self.hx, self.hy, self.lx, self.ly = list(g)
        self.mass = np.zeros(self.size)
        self.trace_mass = np.zeros(self.trace_size)
        L.oracle_mass(ctypes.c_void_p(self.h), _p(self.mass), _p(self.trace_mass))

    def __del__(self):
        if getattr(self, "h", None):
            lib().oracle_destroy(ctypes.c_void_p(self.h))
            self.h = None

    def _call(self, name, *args):
        rc = getattr(lib(), name)(ctypes.c_void_p(self.h), *args)
        if rc != 0:
            raise OracleError(lib().oracle_error().decode())

    def basis(self):
        x, w = np.zeros(self.n), np.zeros(self.n)
        self._call("oracle_basis", _p(x), _p(w))
        return x, w

    def initial(self) -> np.ndarray:
        u = np.zeros(self.size)
        self._call("oracle_initial", _p(u))
        return u

    def exact(self, x, y, t):
        s = np.zeros(4)
        self._call("oracle_exact", ctypes.c_double(x), ctypes.c_double(y), ctypes.c_double(t), _p(s))
        return s

    def freeze(self, u) -> float:
        r = ctypes.c_double()
        self._call("oracle_freeze", _p(np.ascontiguousarray(u)), ctypes.byref(r))
        return r.value

    def speeds(self) -> np.ndarray:
        ab = np.zeros(2 * self.faces * self.n)
        self._call("oracle_speeds", _p(ab))
        return ab.reshape(-1, 2)

    def set_stage(self, old, step: float) -> None:
        self._call("oracle_set_stage", _p(np.ascontiguousarray(old)), ctypes.c_double(step))

    def residual(self, u) -> np.ndarray:
        r = np.zeros(self.size)
        self._call("oracle_residual", _p(np.ascontiguousarray(u)), _p(r))
        return r

    def trace(self, u) -> np.ndarray:
        lam = np.zeros(self.trace_size)
        self._call("oracle_trace", _p(np.ascontiguousarray(u)), _p(lam))
        return lam

    def hybrid_residual(self, u, lam):
        r, g = np.zeros(self.size), np.zeros(self.trace_size)
        self._call("oracle_hybrid_residual", _p(np.ascontiguousarray(u)), _p(np.ascontiguousarray(lam)), _p(r), _p(g))
        return r, g

    def admissible(self, u) -> bool:
        ok = ctypes.c_int()
        self._call("oracle_admissible", _p(np.ascontiguousarray(u)), ctypes.byref(ok))
        return bool(ok.value)

    def integral(self, u) -> np.ndarray:
        s = np.zeros(4)
        self._call("oracle_integral", _p(np.ascontiguousarray(u)), _p(s))
        return s

    def l2_error(self, u, t) -> np.ndarray:
        s = np.zeros(4)
        self._call("oracle_l2_error", _p(np.ascontiguousarray(u)), ctypes.c_double(t), _p(s))
        return s

    def dual_norm(self, r) -> float:
        return float(np.sqrt(np.sum(r * r / self.mass)))

    def rms(self, r) -> float:
        return self.dual_norm(r) / np.sqrt(self.lx * self.ly)

    # DG operator
    def dg_refresh(self, u) -> None:
        self._call("oracle_dg_refresh", _p(np.ascontiguousarray(u)))

    def dg_apply(self, d) -> np.ndarray:
        o = np.zeros(self.size)
        self._call("oracle_dg_apply", _p(np.ascontiguousarray(d)), _p(o))
        return o

    def dg_apply_transpose(self, w) -> np.ndarray:
        o = np.zeros(self.size)
        self._call("oracle_dg_apply_transpose", _p(np.ascontiguousarray(w)), _p(o))
        return o

    def dg_block(self, row: int, col: int) -> np.ndarray:
        """Dense block as a row-major (m, m) array (the reference stores it column-major)."""
        o = np.zeros(self.block * self.block)
        self._call("oracle_dg_block", ctypes.c_int(row), ctypes.c_int(col), _p(o))
        return o.reshape(self.block, self.block).T.copy()

    def trace_diagonal(self) -> np.ndarray:
        o = np.zeros(self.trace_size)
        self._call("oracle_trace_diagonal", _p(o))
        return o

    def dg_precond_refresh(self) -> None:
        self._call("oracle_dg_precond_refresh")

    def dg_precond_refresh_ilu(self) -> None:
        """2D block ILU(0) of the DG Jacobian on the cartesian block graph (GMRES op 2)."""
        self._call("oracle_dg_precond_refresh_ilu")

    def dg_precond_apply_ilu(self, x) -> np.ndarray:
        """z = M^{-1} x with the 2D block ILU(0) factors of dg_precond_refresh_ilu."""
        o = np.zeros(self.size)
        self._call("oracle_dg_precond_apply_ilu", _p(np.ascontiguousarray(x)), _p(o))
        return o

    def dg_precond_apply(self, x) -> np.ndarray:
        o = np.zeros(self.size)
        self._call("oracle_dg_precond_apply", _p(np.ascontiguousarray(x)), _p(o))
        return o

    # HDG operator
    def hdg_refresh(self, u, r) -> None:
        self._call("oracle_hdg_refresh", _p(np.ascontiguousarray(u)), _p(np.ascontiguousarray(r)))

    def hdg_rhs(self) -> np.ndarray:
        o = np.zeros(self.trace_size)
        self._call("oracle_hdg_rhs", _p(o))
        return o

    def hdg_apply(self, d) -> np.ndarray:
        o = np.zeros(self.trace_size)
        self._call("oracle_hdg_apply", _p(np.ascontiguousarray(d)), _p(o))
        return o

    def hdg_block(self, row: int, col: int) -> np.ndarray:
        fw = 4 * self.n
        o = np.zeros(fw * fw)
        self._call("oracle_hdg_block", ctypes.c_int(row), ctypes.c_int(col), _p(o))
        return o.reshape(fw, fw).T.copy()

    def hdg_recover(self, d) -> np.ndarray:
        o = np.zeros(self.size)
        self._call("oracle_hdg_recover", _p(np.ascontiguousarray(d)), _p(o))
        return o

    def hdg_recovered_residual(self, e) -> np.ndarray:
        o = np.zeros(self.size)
        self._call("oracle_hdg_recovered_residual", _p(np.ascontiguousarray(e)), _p(o))
        return o

    def hdg_schur(self) -> np.ndarray:
        t = 16 * self.n
        o = np.zeros(self.cells * t * t)
        self._call("oracle_hdg_schur", _p(o))
        return o.reshape(self.cells, t, t).transpose(0, 2, 1).copy()

    def hdg_precond_refresh(self) -> None:
        self._call("oracle_hdg_precond_refresh")

    def hdg_precond_apply(self, x) -> np.ndarray:
        o = np.zeros(self.trace_size)
        self._call("oracle_hdg_precond_apply", _p(np.ascontiguousarray(x)), _p(o))
        return o

    def gmres(self, op: int, rhs, restart: int, limit: int, tol: float):
        """op 0: DG with block-Jacobi, 1: Schur with face block-Jacobi, 2: DG with 2D block ILU(0)."""
        n = self.trace_size if op == 1 else self.size
        x, res = np.zeros(n), np.zeros(n)
        it, rel = ctypes.c_int(), ctypes.c_double()
        self._call("oracle_gmres", ctypes.c_int(op), ctypes.c_int(restart), _p(np.ascontiguousarray(rhs)),
                   _p(x), ctypes.c_int(limit), ctypes.c_double(tol), ctypes.byref(it), ctypes.byref(rel), _p(res))
        return x, it.value, rel.value, res

    def advance(self, method: str, u, max_updates: int = 4096):
        """Run the time integrator; returns (state, stats dict, updates array [k, 13])."""
        s = np.ascontiguousarray(u, dtype=np.float64).copy()
        stats = np.zeros(8)
        upd = np.zeros(13 * max_updates)
        cnt = ctypes.c_int()
        self._call("oracle_advance", ctypes.c_int(0 if method == "dg" else 1), _p(s), _p(stats), _p(upd),
                   ctypes.c_int(max_updates), ctypes.byref(cnt))
        keys = ["final_time", "conservation_drift", "newton_iterations", "krylov_iterations", "steps",
                "max_linear_residual", "max_dg_linear_residual", "seconds"]
        return s, dict(zip(keys, stats.tolist())), upd[: 13 * min(cnt.value, max_updates)].reshape(-1, 13)


class Oracle1D:
    """One 1D oracle Problem plus its DG and HDG operators (dg_hdg_1d/include/euler/*.hpp).
    Volume vectors are [cell][var][node] with NVAR = 3; trace vectors hold NVAR values per face,
    face e joining cells e and e+1 (periodic)."""

    NVAR = 3

    def __init__(self, args: str):
        L = lib()
        self.h = L.oracle1d_create(args.encode())
        if not self.h:
            raise OracleError(L.oracle_error().decode())
        s = (ctypes.c_longlong * 6)()
        L.oracle1d_sizes(ctypes.c_void_p(self.h), s)
        self.size, self.trace_size, self.block, self.cells, self.n, self.points = (int(x) for x in s)
        self.mass = np.zeros(self.size)
        L.oracle1d_mass(ctypes.c_void_p(self.h), _p(self.mass))

    def __del__(self):
        if getattr(self, "h", None):
            lib().oracle1d_destroy(ctypes.c_void_p(self.h))
            self.h = None

    def _call(self, name, *args):
        rc = getattr(lib(), name)(ctypes.c_void_p(self.h), *args)
        if rc != 0:
            raise OracleError(lib().oracle_error().decode())

    def _vol(self, name, *args):
        o = np.zeros(self.size)
        self._call(name, *[_p(np.ascontiguousarray(a, dtype=np.float64)) for a in args], _p(o))
        return o

    def _tr(self, name, *args):
        o = np.zeros(self.trace_size)
        self._call(name, *[_p(np.ascontiguousarray(a, dtype=np.float64)) for a in args], _p(o))
        return o

    def basis(self):
        """Nodes x, weights w, values [Q, n] and weighted derivatives [Q, n]."""
        x, w = np.zeros(self.n), np.zeros(self.n)
        v, d = np.zeros(self.points * self.n), np.zeros(self.points * self.n)
        self._call("oracle1d_basis", _p(x), _p(w), _p(v), _p(d))
        return x, w, v.reshape(self.points, self.n), d.reshape(self.points, self.n)

    def initial(self) -> np.ndarray:
        u = np.zeros(self.size)
        self._call("oracle1d_initial", _p(u))
        return u

    def exact(self, x, t):
        s = np.zeros(3)
        self._call("oracle1d_exact", ctypes.c_double(x), ctypes.c_double(t), _p(s))
        return s

    def freeze(self, u) -> float:
        r = ctypes.c_double()
        self._call("oracle1d_freeze", _p(np.ascontiguousarray(u)), ctypes.byref(r))
        return r.value

    def speeds(self) -> np.ndarray:
        ab = np.zeros(2 * self.cells)
        self._call("oracle1d_speeds", _p(ab))
        return ab.reshape(-1, 2)

    def set_stage(self, old, step: float) -> None:
        self._call("oracle1d_set_stage", _p(np.ascontiguousarray(old)), ctypes.c_double(step))

    def residual(self, u) -> np.ndarray:
        return self._vol("oracle1d_residual", u)

    def trace(self, u) -> np.ndarray:
        return self._tr("oracle1d_trace", u)

    def admissible(self, u) -> bool:
        ok = ctypes.c_int()
        self._call("oracle1d_admissible", _p(np.ascontiguousarray(u)), ctypes.byref(ok))
        return bool(ok.value)

    def integral(self, u) -> np.ndarray:
        s = np.zeros(3)
        self._call("oracle1d_integral", _p(np.ascontiguousarray(u)), _p(s))
        return s

    def l2_error(self, u, t) -> np.ndarray:
        s = np.zeros(3)
        self._call("oracle1d_l2_error", _p(np.ascontiguousarray(u)), ctypes.c_double(t), _p(s))
        return s

    def dual_norm(self, r) -> float:
        return float(np.sqrt(np.sum(r * r / self.mass)))

    def rms(self, r) -> float:
        return self.dual_norm(r) / np.sqrt(2.0)

    def dg_refresh(self, u) -> None:
        self._call("oracle1d_dg_refresh", _p(np.ascontiguousarray(u)))

    def dg_apply(self, d) -> np.ndarray:
        return self._vol("oracle1d_dg_apply", d)

    def dg_block(self, row: int, col: int) -> np.ndarray:
        """Dense block as a row-major (m, m) array (the reference stores it column-major)."""
        o = np.zeros(self.block * self.block)
        self._call("oracle1d_dg_block", ctypes.c_int(row), ctypes.c_int(col), _p(o))
        return o.reshape(self.block, self.block).T.copy()

    def dg_precond_refresh(self) -> None:
        self._call("oracle1d_dg_precond_refresh")

    def dg_precond_apply_ilu(self, x) -> np.ndarray:
        """z = M^{-1} x with the 2D block ILU(0) factors of dg_precond_refresh_ilu."""
        o = np.zeros(self.size)
        self._call("oracle_dg_precond_apply_ilu", _p(np.ascontiguousarray(x)), _p(o))
        return o

    def dg_precond_apply(self, x) -> np.ndarray:
        return self._vol("oracle1d_dg_precond_apply", x)

    def hdg_refresh(self, u, r) -> None:
        self._call("oracle1d_hdg_refresh", _p(np.ascontiguousarray(u)), _p(np.ascontiguousarray(r)))

    def hdg_rhs(self) -> np.ndarray:
        o = np.zeros(self.trace_size)
        self._call("oracle1d_hdg_rhs", _p(o))
        return o

    def hdg_apply(self, d) -> np.ndarray:
        return self._tr("oracle1d_hdg_apply", d)

    def hdg_block(self, row: int, col: int) -> np.ndarray:
        o = np.zeros(9)
        self._call("oracle1d_hdg_block", ctypes.c_int(row), ctypes.c_int(col), _p(o))
        return o.reshape(3, 3).T.copy()

    def hdg_recover(self, d) -> np.ndarray:
        return self._vol("oracle1d_hdg_recover", d)

    def hdg_recovered_residual(self, dl) -> np.ndarray:
        """The DG residual implied by the Schur error S dl - rhs (hybrid.cpp:118-130)."""
        return self._vol("oracle1d_hdg_recovered_residual", dl)

    def hdg_precond_refresh(self) -> None:
        self._call("oracle1d_hdg_precond_refresh")

    def hdg_precond_apply(self, x) -> np.ndarray:
        return self._tr("oracle1d_hdg_precond_apply", x)

    def gmres(self, op: int, rhs, restart: int, limit: int, tol: float):
        n = self.size if op == 0 else self.trace_size
        x, res = np.zeros(n), np.zeros(n)
        it, rel = ctypes.c_int(), ctypes.c_double()
        self._call("oracle1d_gmres", ctypes.c_int(op), ctypes.c_int(restart), _p(np.ascontiguousarray(rhs)),
                   _p(x), ctypes.c_int(limit), ctypes.c_double(tol), ctypes.byref(it), ctypes.byref(rel), _p(res))
        return x, it.value, rel.value, res

    def advance(self, method: str, u, max_updates: int = 4096):
        """Run the time integrator; returns (state, stats dict, updates array [k, 13])."""
        s = np.ascontiguousarray(u, dtype=np.float64).copy()
        stats = np.zeros(8)
        upd = np.zeros(13 * max_updates)
        cnt = ctypes.c_int()
        self._call("oracle1d_advance", ctypes.c_int(0 if method == "dg" else 1), _p(s), _p(stats), _p(upd),
                   ctypes.c_int(max_updates), ctypes.byref(cnt))
        keys = ["final_time", "conservation_drift", "newton_iterations", "krylov_iterations", "steps",
                "max_linear_residual", "max_dg_linear_residual", "seconds"]
        return s, dict(zip(keys, stats.tolist())), upd[: 13 * min(cnt.value, max_updates)].reshape(-1, 13)


def run_cli(args: list[str], cwd: str | None = None) -> subprocess.CompletedProcess:
    """Run the oracle's reference-compatible CLI (dg_hdg_2d/src/main.cpp flags)."""
    if not CLI_PATH.exists():
        build()
    return subprocess.run([str(CLI_PATH), *args], cwd=cwd, capture_output=True, text=True)


def run_cli_1d(args: list[str], cwd: str | None = None) -> subprocess.CompletedProcess:
    """Run the 1D oracle's reference-compatible CLI (dg_hdg_1d/src/main.cpp flags)."""
    if not CLI1D_PATH.exists():
        build()
    return subprocess.run([str(CLI1D_PATH), *args], cwd=cwd, capture_output=True, text=True)


def ilu_exactness(count: int, width: int, full: bool) -> float:
    """max |x - exact| of one block ILU(0) application on the path (full=False) or full block
    graph of the reference's own check (check_1d.cpp:109-138)."""
    err = ctypes.c_double()
    if lib().oracle_ilu_exactness(count, width, 1 if full else 0, ctypes.byref(err)) != 0:
        raise OracleError(lib().oracle_error().decode())
    return err.value
