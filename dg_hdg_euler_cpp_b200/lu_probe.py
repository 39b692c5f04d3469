"""Phase split of the left-looking LU kernels (k_lu_left) from the cycle-counter build.

    make -C dg_hdg_euler_cpp_b200/csrc probe      # lib/libdgh_gpu_probe.so (csrc/lu_probe.h)
    python -m dg_hdg_euler_cpp_b200.lu_probe --nx 64 --k 8 --precision mixed

Runs one block-Jacobi refresh (DG: k_dg_assemble + k_lu_left<false>) and one HDG condensation
(k_hdg_assemble + k_lu_left<true> + k_hdg_schur) on the initial state, each once to warm up and
once counted, and prints per kernel the share of thread 0's cycles in each phase of the kernel
(LL_PROBE hooks in dgh_kernels_lu2.cuh), with the mean cycles per CTA.  The counters add a few
instructions per column to thread 0: use the shares, not the times, and time the kernels with
the ordinary build (bench.py).
"""
from __future__ import annotations

import argparse
import ctypes

import numpy as np

from . import _lib

PROBE_LIB = _lib.PKG / "lib" / "libdgh_gpu_probe.so"
PHASES = {0: "panel load", 1: "chunk triangle", 2: "chunk GEMM", 3: "pivot search", 7: "elimination",
          6: "rank-4 update", 4: "write-back + inverses", 5: "right-hand sides / final layout"}


def phase_split(lib, run) -> tuple[dict[str, float], float, int]:
    """Shares per phase, mean cycles per CTA and CTA count of the k_lu_left launches in run()."""
    run()  # warm-up: the first call also tunes launch attributes
    table = (ctypes.c_ulonglong * (1024 * 8))()
    if lib.ll_probe_reset() != 0:
        raise RuntimeError("ll_probe_reset failed")
    run()
    if lib.ll_probe_read(table) != 0:
        raise RuntimeError("ll_probe_read failed")
    a = np.array(table, dtype=np.float64).reshape(1024, 8)
    per_cta = a.sum(1)
    used = per_cta > 0
    total = a.sum(0)
    return ({name: float(total[p] / total.sum()) for p, name in PHASES.items()}, float(per_cta[used].mean()),
            int(used.sum()))


def main(argv=None) -> None:
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--nx", type=int, default=64)
    ap.add_argument("--k", type=int, default=8)
    ap.add_argument("--precision", choices=["fp64", "mixed"], default="mixed")
    a = ap.parse_args(argv)
    lib = _lib.load(PROBE_LIB)
    lib.ll_probe_reset.restype = ctypes.c_int
    lib.ll_probe_read.restype = ctypes.c_int
    lib.ll_probe_read.argtypes = [ctypes.c_void_p]
    from .solver import Solver

    s = Solver(nx=a.nx, ny=a.nx, k=a.k, cfl=5.0, integrator="be", steps=1, method="both", precision=a.precision)
    u = s.initial()
    s.freeze(u)
    s.set_stage(u, .01)
    s.dg_refresh(u)
    r = s.residual(u)
    for tag, run in (("k_lu_left<false> (DG block-Jacobi factors)", lambda: s.precond_refresh("dg")),
                     ("k_lu_left<true> (HDG condensation)", lambda: s.hdg_refresh_projected(u, r))):
        shares, cycles, ctas = phase_split(lib, run)
        print(f"{tag}, {a.nx}x{a.nx} k={a.k} {a.precision}: {ctas} CTAs, {cycles / 1e6:.2f} M cycles per CTA")
        for name, v in shares.items():
            print(f"  {name:32s} {100 * v:5.1f} %")
    s.close()


if __name__ == "__main__":
    main()
