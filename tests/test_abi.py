"""CPU-side checks of the C ABI library: it builds for sm_100a, loads, and exports every entry
point include/dgh_gpu.h declares; without a GPU, context creation fails with an error code
instead of falling back to the CPU."""
import ctypes
import re

import pytest

from conftest import ROOT

HEADER = ROOT / "include" / "dgh_gpu.h"


def declared_functions():
    text = re.sub(r"/\*.*?\*/", "", HEADER.read_text(), flags=re.S)
    names = re.findall(r"\b(dgh_[A-Za-z0-9_]+)\s*\(", text)
    return sorted(set(names))


@pytest.fixture(scope="module")
def lib():
    from dg_hdg_euler_cpp_b200 import _lib

    if not _lib.LIB_PATH.exists():
        _lib.build()
    return _lib.load()


def test_library_exports_every_declared_symbol(lib):
    names = declared_functions()
    assert len(names) >= 45
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_library_exports_nothing_undeclared():
    """Every extern "C" dgh_* symbol the library exports is declared in the header (no hidden
    entry points)."""
    import subprocess

    from dg_hdg_euler_cpp_b200 import _lib

    out = subprocess.run(["nm", "-D", "--defined-only", str(_lib.LIB_PATH)], capture_output=True, text=True,
                         check=True).stdout
    exported = {parts[-1] for parts in (line.split() for line in out.splitlines())
                if len(parts) >= 3 and parts[1] == "T" and parts[-1].startswith("dgh_")}
    assert exported and exported <= set(declared_functions()), sorted(exported - set(declared_functions()))


def test_python_binding_covers_the_header():
    from dg_hdg_euler_cpp_b200 import _lib

    assert set(declared_functions()) == set(_lib.SIGNATURES)


def test_config_defaults_match_reference(lib):
    from dg_hdg_euler_cpp_b200 import _lib

    cfg = _lib.dgh_config()
    lib.dgh_config_default(ctypes.byref(cfg))
    # dg_hdg_2d/include/euler/config.hpp:7-18
    assert (cfg.nx, cfg.ny, cfg.degree, cfg.quadrature) == (8, 8, 3, 0)
    assert (cfg.restart, cfg.max_linear, cfg.max_newton, cfg.steps) == (30, 1500, 30, 0)
    assert (cfg.cfl, cfg.final_time, cfg.safety) == (2.0, 0.2, 1.1)
    assert cfg.nonlinear_tolerance == cfg.linear_tolerance == 1e-12


def test_invalid_configuration_is_rejected_before_any_device_work(lib):
    from dg_hdg_euler_cpp_b200 import _lib

    cfg = _lib.dgh_config()
    lib.dgh_config_default(ctypes.byref(cfg))
    cfg.degree = 9  # config.cpp:7 allows k <= 8
    h = ctypes.c_void_p()
    rc = lib.dgh_ctx_create(ctypes.byref(cfg), ctypes.byref(h))
    assert rc == 1 and not h.value
    assert b"Invalid mesh or degree" in lib.dgh_last_error(None)


@pytest.mark.parametrize("fields,message", [
    ({"dim": 3}, "Invalid dimension"),
    ({"dim": 1, "nx": 2}, "Invalid mesh or degree"),
    ({"dim": 1, "degree": 3, "quadrature": 3}, "Quadrature must be >= degree+1"),
    ({"dim": 1, "degree": 3, "quadrature": 21}, "Quadrature above 20 points"),
    ({"dim": 2, "degree": 3, "quadrature": 17}, "Quadrature above 16 points is not supported on the device (2D)"),
])
def test_dimension_and_quadrature_validation(lib, fields, message):
    """dg_hdg_1d/src/config.cpp:6-21 and the device limits, checked before any device work."""
    from dg_hdg_euler_cpp_b200 import _lib

    cfg = _lib.dgh_config()
    lib.dgh_config_default(ctypes.byref(cfg))
    assert cfg.dim == 2
    for k, v in fields.items():
        setattr(cfg, k, v)
    h = ctypes.c_void_p()
    assert lib.dgh_ctx_create(ctypes.byref(cfg), ctypes.byref(h)) == 1 and not h.value
    assert message.encode() in lib.dgh_last_error(None)


def test_1d_cli_validates_flags_before_device_work():
    """The 1D front end parses dg_hdg_1d's flags and refuses the paths it does not build
    (the block COLAMD ordering, the dense direct solve)."""
    import subprocess

    from dg_hdg_euler_cpp_b200 import BIN1D_PATH

    if not BIN1D_PATH.exists():
        pytest.skip("dgh1d not built")
    for args, msg in [(["--precond", "block-ilu0", "--ordering", "colamd"], "natural block ordering only"),
                      (["--linear", "direct"], "CPU-only"),
                      (["--T", ".1", "--steps", "2"], "Choose either --T or --steps"),
                      (["--integrator", "rk4"], "Invalid integrator"), (["--bogus"], "Unknown option")]:
        res = subprocess.run([str(BIN1D_PATH), *args], capture_output=True, text=True, timeout=60)
        assert res.returncode == 1 and msg in res.stderr, (args, res.stderr)


def test_2d_cli_validates_flags_before_device_work():
    """The 2D front end parses dg_hdg_2d's flags with the reference's texts (config.cpp:23-122):
    block-jacobi is the reference's only 2D preconditioner (block-ilu0 is this front end's DG-only
    extension, natural ordering), and the dense direct solve stays a CPU check."""
    import subprocess

    from dg_hdg_euler_cpp_b200 import BIN_PATH

    if not BIN_PATH.exists():
        pytest.skip("dgh2d not built")
    for args, msg in [(["--precond", "block-ilu1"], "2D currently supports block-jacobi only"),
                      (["--precond", "block-ilu0"], "DG operator only"),
                      (["--precond", "block-ilu0", "--method", "dg", "--ordering", "colamd"], "natural block ordering"),
                      (["--linear", "direct"], "CPU-only"), (["--ordering", "rcm"], "Invalid ordering"),
                      (["--T", ".1", "--steps", "2"], "Choose either --T or --steps"),
                      (["--integrator", "rk4"], "Invalid integrator"), (["--testcase", "vortex"], "Invalid testcase"),
                      (["--method", "fem"], "Method must be dg, hdg, or both"),
                      (["--precision", "fp16"], "Invalid precision"), (["--bogus"], "Unknown option")]:
        res = subprocess.run([str(BIN_PATH), *args], capture_output=True, text=True, timeout=60)
        assert res.returncode == 1 and msg in res.stderr, (args, res.stderr)


def test_no_cpu_fallback_without_gpu(lib):
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from dg_hdg_euler_cpp_b200 import _lib

    cfg = _lib.dgh_config()
    lib.dgh_config_default(ctypes.byref(cfg))
    h = ctypes.c_void_p()
    rc = lib.dgh_ctx_create(ctypes.byref(cfg), ctypes.byref(h))
    assert rc == 2 and not h.value  # DGH_ERR_CUDA


def test_kernels_are_built_for_sm100a():
    log = (ROOT / "dg_hdg_euler_cpp_b200" / "lib" / "ptxas.log").read_text()
    assert "sm_100a" in log
    assert "k_lu" in log and "k_dg_apply" in log and "k_hdg_apply" in log


def test_batch_rejects_members_without_a_single_method(lib):
    from dg_hdg_euler_cpp_b200 import _lib

    cfgs = (_lib.dgh_config * 2)()
    for c in cfgs:
        lib.dgh_config_default(ctypes.byref(c))
        c.method = 0
    cfgs[1].method = 2  # both: a batch member runs one method
    h = ctypes.c_void_p()
    assert lib.dgh_batch_create(cfgs, 2, ctypes.byref(h)) == 1
    assert not h.value
    assert "batch member" in lib.dgh_batch_error(None, 0).decode()
    assert lib.dgh_batch_create(cfgs, 0, ctypes.byref(h)) == 1


def test_uneven_batch_workload_draws():
    """The 16-member uneven batch (seeds 0-15, SplitMix64): degree, mesh, method and amplitude."""
    from dg_hdg_euler_cpp_b200.solver import batch_member

    draws = [batch_member(s) for s in range(16)]
    got = [(d["config"]["k"], d["config"]["nx"], d["config"]["method"]) for d in draws]
    assert got == [(8, 32, "dg"), (4, 128, "hdg"), (6, 96, "dg"), (4, 64, "hdg"), (6, 32, "dg"), (6, 32, "hdg"),
                   (2, 64, "dg"), (8, 32, "hdg"), (6, 64, "dg"), (2, 96, "dg"), (6, 96, "dg"), (4, 64, "dg"),
                   (8, 128, "hdg"), (8, 64, "hdg"), (6, 96, "dg"), (4, 32, "hdg")]
    assert all(0.05 <= d["amplitude"] < 0.25 for d in draws)
    assert abs(draws[0]["amplitude"] - 0.0553) < 1e-4
    # SplitMix64 known answer for state 0 (Vigna's reference generator)
    from dg_hdg_euler_cpp_b200.solver import splitmix64

    assert splitmix64(0)[0] == 0xE220A8397B1DCDAF


def test_perturbation_keeps_states_positive():
    import numpy as np

    from dg_hdg_euler_cpp_b200.solver import perturb

    u = np.ones(3 * 2 * 4 * 9)
    p = perturb(u, 3, 2, 2, 0.25)
    assert p.min() >= 0.75 - 1e-12 and p.max() <= 1.25 + 1e-12
    assert not np.allclose(p, 1)


def test_reference_executable_names():
    """The reference's drivers accept only bin/*.exe (scripts/experiment.py:74-79): the front
    ends are also installed as dg_hdg_2d.exe and dg_hdg.exe (the reference's target names,
    dg_hdg_2d/CMakeLists.txt:16, dg_hdg_1d/CMakeLists.txt:18 with CMAKE_EXECUTABLE_SUFFIX .exe)."""
    import subprocess

    from dg_hdg_euler_cpp_b200 import BIN_PATH

    for name, dim in (("dg_hdg_2d.exe", "2D"), ("dg_hdg.exe", "1D")):
        exe = BIN_PATH.parent / name
        if not exe.exists():
            pytest.skip("front ends not built")
        res = subprocess.run([str(exe), "--help"], capture_output=True, text=True, timeout=60)
        assert res.returncode == 0 and res.stdout.startswith(dim), (name, res.stdout[:80])


def test_library_path_is_exclusive_per_process(lib):
    """A process keeps the library it loaded first: asking for another build of the C ABI after
    the first load is refused."""
    from dg_hdg_euler_cpp_b200 import _lib

    with pytest.raises(RuntimeError, match="already loaded"):
        _lib.load(_lib.LIB_PATH.with_name("libdgh_gpu_other.so"))
    assert _lib.load(_lib.LIB_PATH) is lib
