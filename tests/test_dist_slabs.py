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


def halo_plan(nx, k, rows, above, trace):
    from dg_hdg_euler_cpp_b200 import _lib

    regions, counts = (ctypes.c_int64 * 16)(), (ctypes.c_int * 4)()
    assert _lib.load().dgh_slab_halo_plan(nx, k, rows, above, trace, regions, counts) == 0
    out, i = [], 0
    for c in counts:
        out.append([(regions[i + 2 * j], regions[i + 2 * j + 1]) for j in range(c)])
        i += 2 * c
    return dict(zip(("to_below", "to_above", "from_above", "from_below"), out))


def unit_rows(regions, unit, half):
    """(axis, local row) of every row-sized unit the regions cover; axis 0 for x faces or cells,
    1 for y faces (offsets at or beyond `half`)."""
    rows = []
    for off, cnt in regions:
        assert off % unit == 0 and cnt % unit == 0
        for u in range(off // unit, (off + cnt) // unit):
            rows.append((1, u - half // unit) if half and off >= half else (0, u))
    return rows


@pytest.mark.parametrize("ny,size", [(6, 2), (9, 3), (12, 4), (7, 2), (16, 8)])
@pytest.mark.parametrize("k", [1, 3, 8])
def test_trace_halo_brings_every_face_the_owned_schur_rows_read(ny, size, k):
    """The HDG slab layout against the periodic grid: the Schur apply of an owned face reads the
    faces of the two cells beside it, the recovery of an interior cell its own four faces; each of
    those is owned or arrives by the trace halo, every region received holds the same global
    faces the neighbour sends, and every face sent is owned by its sender."""
    from dg_hdg_euler_cpp_b200.solver import slab_rows

    nx, above, n = 5, 2, k + 1
    fw = 4 * n
    fr = nx * fw
    parts = [slab_rows(ny, size, r) for r in range(size)]
    plans = [halo_plan(nx, k, p[1], above, 1) for p in parts]
    for r, (row0, rows, below, above_rank) in enumerate(parts):
        L = rows + 1 + above
        cells = nx * L
        half = cells * fw

        def nb(cell, side):
            x, y = cell % nx, cell // nx
            if side < 2:
                x = (x + (-1 if side == 0 else 1)) % nx
            else:
                y = (y + (-1 if side == 2 else 1)) % L
            return x + nx * y

        def face_of(cell, side):
            return [nb(cell, 0), cell, cells + nb(cell, 2), cells + cell][side]

        owned = {f for f in range(2 * cells) if 1 <= (f % cells) // nx <= rows}
        got = set(owned)
        for off, cnt in plans[r]["from_above"] + plans[r]["from_below"]:
            got |= set(range(off // fw, (off + cnt) // fw))
        for f in owned:
            axis, first = f // cells, f % cells
            for cell in (first, nb(first, 2 * axis + 1)):
                for side in range(4):
                    assert face_of(cell, side) in got, (r, f, cell, side)
        # the recovery and the recovered residual of an interior cell read its four faces
        for cell in range(nx, nx * (rows + 1)):
            assert all(face_of(cell, side) in got for side in range(4)), (r, cell)

        def global_rows(rank, regions, cells_r):
            row0_r = parts[rank][0]
            return [(a, (row0_r - 1 + j) % ny) for a, j in unit_rows(regions, fr, cells_r * fw)]

        cells_above = nx * (parts[above_rank][1] + 1 + above)
        cells_below = nx * (parts[below][1] + 1 + above)
        assert global_rows(r, plans[r]["from_above"], cells) == global_rows(above_rank, plans[above_rank]["to_below"],
                                                                            cells_above)
        assert global_rows(r, plans[r]["from_below"], cells) == global_rows(below, plans[below]["to_above"],
                                                                            cells_below)
        for off, cnt in plans[r]["to_below"] + plans[r]["to_above"]:
            assert set(range(off // fw, (off + cnt) // fw)) <= owned


@pytest.mark.parametrize("ny,size,above", [(6, 2, 1), (9, 3, 1), (5, 5, 1), (12, 4, 2), (7, 3, 2)])
def test_volume_halo_fills_every_ghost_row_with_the_right_global_row(ny, size, above):
    from dg_hdg_euler_cpp_b200.solver import slab_rows

    nx, k = 4, 2
    rl = nx * 4 * (k + 1) ** 2
    parts = [slab_rows(ny, size, r) for r in range(size)]
    if min(p[1] for p in parts) < above:
        pytest.skip("fewer rows than ghost rows above")
    plans = [halo_plan(nx, k, p[1], above, 0) for p in parts]
    for r, (row0, rows, below, up) in enumerate(parts):
        filled = {j for off, cnt in plans[r]["from_above"] + plans[r]["from_below"]
                  for j in range(off // rl, (off + cnt) // rl)}
        assert filled == {0} | set(range(rows + 1, rows + 1 + above))  # every ghost row, nothing else

        def g(rank, regions):
            return [(parts[rank][0] - 1 + j) % ny for _, j in unit_rows(regions, rl, 0)]

        assert g(r, plans[r]["from_above"]) == g(up, plans[up]["to_below"])
        assert g(r, plans[r]["from_below"]) == g(below, plans[below]["to_above"])
        for off, cnt in plans[r]["to_below"] + plans[r]["to_above"]:
            assert all(1 <= j <= rows for j in range(off // rl, (off + cnt) // rl))


def test_halo_plan_rejects_bad_shapes():
    from dg_hdg_euler_cpp_b200 import _lib

    regions, counts = (ctypes.c_int64 * 16)(), (ctypes.c_int * 4)()
    lib = _lib.load()
    for args in ((4, 2, 1, 2, 1), (4, 9, 3, 1, 0), (0, 2, 3, 1, 0), (4, 2, 3, 3, 1)):
        assert lib.dgh_slab_halo_plan(*args, regions, counts) == 1
