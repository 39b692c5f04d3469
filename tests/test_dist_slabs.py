"""Host side of the slab domain decomposition (dgh_slab_rows, dgh_comm_*, dgh_ctx_create_slab),
on CPU: the row partition every rank computes on its own, the refusals of configurations the
decomposition does not cover (before any device work), the in-process group's handles, and the
NCCL id made on rank 0 and shared over a torch.distributed group of two gloo ranks, whose ranks
then agree on a partition that covers the mesh once."""
import ctypes
import os
import subprocess
import sys

import pytest

from conftest import ROOT
from test_dist_replicas import free_port


def test_partition_covers_every_row_once():
    from dg_hdg_euler_cpp_b200.solver import slab_rows

    for ny in range(3, 41):
        for size in range(1, min(ny, 9) + 1):
            parts = [slab_rows(ny, size, r) for r in range(size)]
            rows = [p[1] for p in parts]
            assert sum(rows) == ny and max(rows) - min(rows) <= 1 and min(rows) >= 1
            nxt = 0
            for r, (row0, n, below, above) in enumerate(parts):
                assert row0 == nxt
                nxt += n
                assert below == (r - 1) % size and above == (r + 1) % size
            assert nxt == ny


def test_partition_rejects_more_ranks_than_rows():
    from dg_hdg_euler_cpp_b200.solver import DGHError, slab_rows

    for args in ((4, 5, 0), (8, 2, 2), (8, 0, 0), (8, 2, -1)):
        with pytest.raises(DGHError):
            slab_rows(*args)


def test_slab_context_refuses_uncovered_configurations():
    """Refused before any device call, so these run without a GPU."""
    from dg_hdg_euler_cpp_b200 import _lib
    from dg_hdg_euler_cpp_b200.solver import SlabComm, make_config

    lib = _lib.load()
    comms = SlabComm.local_group(2)
    cases = [(dict(method="both"), "2D DG or HDG method"), (dict(dim=1, cells=12), "2D DG or HDG method"),
             (dict(quad=6, k=3), "collocated volume rule"), (dict(precond="block-ilu0"), "block-Jacobi"),
             (dict(method="hdg", ny=3), "two mesh rows per rank")]
    for kw, msg in cases:
        base = dict(nx=8, ny=8, k=3, method="dg")
        base.update(kw)
        cfg = make_config(**base)
        out = ctypes.c_void_p()
        assert lib.dgh_ctx_create_slab(ctypes.byref(cfg), comms[0].h, ctypes.byref(out)) == 1
        assert msg in lib.dgh_last_error(None).decode()
    cfg = make_config(nx=8, ny=8, k=3, method="dg")
    assert lib.dgh_ctx_create_slab(ctypes.byref(cfg), None, ctypes.byref(ctypes.c_void_p())) == 1
    big = SlabComm.local_group(9)
    cfg = make_config(nx=8, ny=8, k=3, method="dg")
    assert lib.dgh_ctx_create_slab(ctypes.byref(cfg), big[0].h, ctypes.byref(ctypes.c_void_p())) == 1
    assert "one mesh row per rank" in lib.dgh_last_error(None).decode()
    for c in comms + big:
        c.close()


def test_local_group_handles():
    from dg_hdg_euler_cpp_b200 import _lib
    from dg_hdg_euler_cpp_b200.solver import DGHError, SlabComm

    g = SlabComm.local_group(3, timeout_ms=500)
    assert [(c.rank, c.size, c.kind) for c in g] == [(0, 3, "local"), (1, 3, "local"), (2, 3, "local")]
    g[0].set_timeout(2000)
    with pytest.raises(DGHError):
        g[0].set_timeout(0)
    g[1].fail("host-side failure")  # marks the group failed; needs no device
    for c in g:
        c.close()
    with pytest.raises(DGHError, match="invalid group size"):
        SlabComm.local_group(0)
    assert _lib.load().dgh_comm_info(None, (ctypes.c_int * 3)()) == 1


WORKER = r"""
import json, sys
sys.path.insert(0, sys.argv[1])
import torch
import torch.distributed as dist
from dg_hdg_euler_cpp_b200.solver import share_unique_id, slab_rows
dist.init_process_group("gloo", init_method="env://")
rank, world = dist.get_rank(), dist.get_world_size()
uid = share_unique_id()
ids = [None] * world
dist.all_gather_object(ids, uid.hex())
parts = [None] * world
dist.all_gather_object(parts, slab_rows(int(sys.argv[2]), world, rank))
print(json.dumps({"rank": rank, "len": len(uid), "same": len(set(ids)) == 1, "parts": parts}))
dist.destroy_process_group()
"""


@pytest.mark.parametrize("ny", [5, 64])
def test_two_gloo_ranks_share_the_nccl_id_and_partition(ny):
    import json

    port = free_port()
    procs = []
    for rank in range(2):
        env = dict(os.environ, RANK=str(rank), WORLD_SIZE="2", MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port),
                   CUDA_VISIBLE_DEVICES="")
        procs.append(subprocess.Popen([sys.executable, "-c", WORKER, str(ROOT), str(ny)], env=env,
                                      stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True))
    rows = []
    for p in procs:
        out, err = p.communicate(timeout=300)
        assert p.returncode == 0, err[-2000:]
        rows.append(json.loads(out.strip().splitlines()[-1]))
    assert sorted(r["rank"] for r in rows) == [0, 1]
    for r in rows:
        assert r["len"] == 128 and r["same"]
        parts = r["parts"]
        assert parts[0][0] == 0 and parts[0][0] + parts[0][1] == parts[1][0] and parts[1][0] + parts[1][1] == ny
