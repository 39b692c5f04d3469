"""The multi-process plumbing of bench.py (one process per GPU, replicas only): two gloo ranks on
CPU take the same barriers and reduce each timing to the maximum over ranks; the reference arm
prints from rank 0 only."""
import os
import socket
import subprocess
import sys

import pytest

from conftest import ROOT


def free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


WORKER = r"""
import os, sys, json
sys.path.insert(0, sys.argv[1])
import torch
import bench
rank, local, world, pg = bench.dist_setup(2, backend="gloo")
bench.barrier(pg, torch)
got = bench.allmax(pg, torch, 10.0 + 5.0 * rank)
bench.barrier(pg, torch)
print(json.dumps({"rank": rank, "world": world, "max": got}))
pg.destroy_process_group()
"""


def run_ranks(code, extra_env=None, args=()):
    port = free_port()
    procs = []
    for rank in range(2):
        env = dict(os.environ, RANK=str(rank), LOCAL_RANK=str(rank), WORLD_SIZE="2", MASTER_ADDR="127.0.0.1",
                   MASTER_PORT=str(port), CUDA_VISIBLE_DEVICES="", **(extra_env or {}))
        procs.append(subprocess.Popen([sys.executable, "-c", code, str(ROOT), *args], env=env, stdout=subprocess.PIPE,
                                      stderr=subprocess.PIPE, text=True))
    outs = []
    for p in procs:
        out, err = p.communicate(timeout=300)
        assert p.returncode == 0, err[-2000:]
        outs.append(out)
    return outs


def test_two_gloo_ranks_take_the_max_over_ranks():
    import json

    outs = run_ranks(WORKER)
    rows = [json.loads(o.strip().splitlines()[-1]) for o in outs]
    assert sorted(r["rank"] for r in rows) == [0, 1]
    assert all(r["world"] == 2 and r["max"] == 15.0 for r in rows)


def test_reference_arm_prints_on_rank_zero_only():
    code = r"""
import sys
sys.path.insert(0, sys.argv[1])
import bench
sys.argv = ["bench.py", "--impl", "reference", "--gpus", "2", "--steps", "2", "--warmup", "1", "--nx", "256",
            "--k", "2"]
bench.main()
"""
    outs = run_ranks(code)
    lines = [[l for l in o.splitlines() if l.startswith("{")] for o in outs]
    assert len(lines[0]) == 1 and lines[1] == []
    assert '"impl": "reference"' in lines[0][0]
    import json

    rec = json.loads(lines[0][0])
    assert rec["value"] > 0 and rec["config"]["proxy_mesh"] == "16x16" and rec["config"]["cell_ratio"] == 256
    assert rec["cpu_baseline"]["cores"] >= 1 and rec["cpu_baseline"]["host"]["nproc"] >= 1
    assert rec["cpu_baseline"]["per_method"]["dg"]["krylov"]


def test_protocol_units_time_updates_two_to_four_only():
    """K timed updates come in ceil(K/3) protocol units of at most 3 (updates 2-4 of each unit)."""
    import bench

    assert bench.protocol_units(20) == [3, 3, 3, 3, 3, 3, 2]
    assert bench.protocol_units(3) == [3]
    assert bench.protocol_units(1) == [1]
    assert sum(bench.protocol_units(17)) == 17 and max(bench.protocol_units(17)) == 3


def test_roofline_peaks_file(tmp_path):
    """bench.py takes the measured copy bandwidth from the measured peaks file when it holds one
    and says so; a missing, unreadable or incomplete file gives the fallback figures."""
    import json

    from conftest import ROOT

    sys.path.insert(0, str(ROOT))
    import bench

    f = tmp_path / "MEASURED_PEAKS.json"
    assert bench.load_peaks(f) == (bench.FALLBACK_PEAKS, "fallback")
    f.write_text(json.dumps({"hbm_gbs": 6547.5, "bf16_tflops": 1500.0, "clocks": {"sm": 1965}}))
    peaks, src = bench.load_peaks(f)
    assert src == "measured" and peaks["hbm_gbs"] == 6547.5 and peaks["bf16_tflops"] == 1500.0
    for bad in ("{", json.dumps({"bf16_tflops": 1500.0}), json.dumps({"hbm_gbs": None}), json.dumps({"hbm_gbs": 0})):
        f.write_text(bad)
        assert bench.load_peaks(f) == (bench.FALLBACK_PEAKS, "fallback"), bad


def test_roofline_bytes_and_traffic_at_the_bench_mesh():
    """The per-launch algorithmic bytes of the dominant kernels at 256^2 k = 8 (m = 324, fw = 36,
    t = 144), and the DRAM traffic the line reports, scaled from the 64^2 captures."""
    import types

    sys.path.insert(0, str(ROOT))
    import bench

    E, m, fw, t = 256 * 256, 324, 36, 144
    assert abs(bench.algorithmic_bytes("dg", m, E, fw, 2 * E, t, "mixed16") - 14.439e9) < 0.01e9
    assert abs(bench.algorithmic_bytes("dg", m, E, fw, 2 * E, t, "mixed") - 27.94e9) < 0.01e9
    assert abs(bench.algorithmic_bytes("dg", m, E, fw, 2 * E, t, "fp64") - 55.46e9) < 0.01e9
    assert abs(bench.algorithmic_bytes("hdg_schur", m, E, fw, 2 * E, t, "mixed") - 5.55e9) < 0.01e9
    args = types.SimpleNamespace(k=8, nx=256)
    half, src = bench.solve_traffic(args, "k_lu_solve_half (block-Jacobi solve from FP16 slabs)")
    assert 1.0 < half / bench.algorithmic_bytes("dg", m, E, fw, 2 * E, t, "mixed16") < 1.1 and "profiles/" in src
    fp32, _ = bench.solve_traffic(args, "k_lu_solve<float> (block-Jacobi solve)")
    assert 1.0 < fp32 / bench.algorithmic_bytes("dg", m, E, fw, 2 * E, t, "mixed") < 1.05
    assert bench.solve_traffic(args, "k_hdg_apply32 (Schur apply)") == (None, None)
    assert bench.solve_traffic(types.SimpleNamespace(k=4, nx=256), "k_lu_solve_half") == (None, None)
