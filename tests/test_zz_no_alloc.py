"""The allocation-free residual entry point against the regular one.

dgh_residual_noalloc serves callers that cannot allocate device memory (an allocation-free
time loop, work issued during CUDA-graph capture, hosts that plan all device memory): it keeps
its only scratch, the face restrictions of u, in a fixed device array inside the library.  Here
it is called through the C ABI twice in a row, on different states, and each result must match
dgh_residual (which uses a context-allocated scratch buffer) to the residual tolerance used by the
parity tests.  This file is collected last so that a failure here never hides another test.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

RTOL = 1e-12  # the residual tolerance of tests/test_gpu_parity.py


def direction(n):
    i = np.arange(n)
    return .2 * np.sin(.31 * i) + .1 * np.cos(.79 * i)


@pytest.mark.parametrize("nx,ny,k,testcase", [(12, 10, 4, "diagonal"), (9, 9, 8, "diagonal"), (7, 5, 2, "wave")])
def test_noalloc_residual_matches_regular_entry_point_twice(nx, ny, k, testcase):
    import torch

    from dg_hdg_euler_cpp_b200.solver import TESTCASES, Solver

    s = Solver(nx=nx, ny=ny, k=k, cfl=1.0, integrator="be", steps=1, method="dg", testcase=testcase)
    u0 = s.initial()
    s.freeze(u0)
    dt = 0.01
    s.set_stage(u0, dt)
    speeds = torch.as_tensor(s.speeds().reshape(-1).copy(), device=s.device)
    errbuf = ctypes.create_string_buffer(256)
    states = [u0 + 1e-3 * s.tensor(direction(s.size)), u0 - 2e-3 * s.tensor(direction(s.size)[::-1].copy())]
    outs = []
    for u in states:  # two calls in a row on different inputs
        r = torch.full_like(u, float("nan"))
        torch.cuda.synchronize()
        rc = s.lib.dgh_residual_noalloc(nx, ny, k, TESTCASES[testcase], ctypes.c_double(dt),
                                        ctypes.c_void_p(u.data_ptr()), ctypes.c_void_p(u0.data_ptr()),
                                        ctypes.c_void_p(speeds.data_ptr()), ctypes.c_void_p(r.data_ptr()),
                                        None, errbuf, len(errbuf))
        assert rc == 0, errbuf.value.decode()
        torch.cuda.synchronize()
        outs.append(r.cpu().numpy())
    for u, got in zip(states, outs):
        ref = s.residual(u).cpu().numpy()
        assert np.all(np.isfinite(got))
        assert np.max(np.abs(got - ref)) <= RTOL * np.max(np.abs(ref))
    s.close()


def test_noalloc_rejects_meshes_beyond_its_scratch():
    import torch

    from dg_hdg_euler_cpp_b200 import _lib

    lib = _lib.load()
    buf = torch.zeros(8, dtype=torch.float64, device="cuda")
    p = ctypes.c_void_p(buf.data_ptr())
    errbuf = ctypes.create_string_buffer(256)
    # 200 x 200 cells at k = 8 need 5.76e6 doubles of traces, beyond the 2,097,152 capacity;
    # the call must refuse before touching any pointer
    rc = lib.dgh_residual_noalloc(200, 200, 8, 0, ctypes.c_double(0.01), p, p, p, p, None, errbuf, len(errbuf))
    assert rc == 1
    assert b"too large" in errbuf.value and b"2097152" in errbuf.value


def test_noalloc_residual_inside_cuda_graph_capture():
    """The use the entry point exists for: after one warm call (which looks up the scratch
    address), one call is captured into a CUDA graph on torch's capture stream; the graph is then
    replayed on two states copied into the captured input buffer, and each replay must match
    dgh_residual."""
    import torch

    from dg_hdg_euler_cpp_b200.solver import TESTCASES, Solver

    nx, ny, k = 10, 8, 5
    s = Solver(nx=nx, ny=ny, k=k, cfl=1.0, integrator="be", steps=1, method="dg", testcase="diagonal")
    u0 = s.initial()
    s.freeze(u0)
    dt = 0.02
    s.set_stage(u0, dt)
    speeds = torch.as_tensor(s.speeds().reshape(-1).copy(), device=s.device)
    errbuf = ctypes.create_string_buffer(256)
    u_in = u0.clone()
    r_out = torch.full_like(u0, float("nan"))

    def call(stream):
        return s.lib.dgh_residual_noalloc(nx, ny, k, TESTCASES["diagonal"], ctypes.c_double(dt),
                                          ctypes.c_void_p(u_in.data_ptr()), ctypes.c_void_p(u0.data_ptr()),
                                          ctypes.c_void_p(speeds.data_ptr()), ctypes.c_void_p(r_out.data_ptr()),
                                          stream, errbuf, len(errbuf))

    assert call(None) == 0, errbuf.value.decode()  # warm call before the capture
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    side = torch.cuda.Stream()
    with torch.cuda.graph(g, stream=side):
        rc = call(ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert rc == 0, errbuf.value.decode()
    states = [u0 + 1e-3 * s.tensor(direction(s.size)), u0 - 3e-3 * s.tensor(direction(s.size)[::-1].copy())]
    for u in states:
        u_in.copy_(u)
        r_out.fill_(float("nan"))
        g.replay()
        torch.cuda.synchronize()
        got = r_out.cpu().numpy()
        ref = s.residual(u).cpu().numpy()
        assert np.all(np.isfinite(got))
        assert np.max(np.abs(got - ref)) <= RTOL * np.max(np.abs(ref))
    del g
    s.close()
