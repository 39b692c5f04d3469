#!/usr/bin/env python3
"""Copy the reference's archived result CSVs used as golden vectors into tests/golden/.

The reference (YueWu2002/DG_HDG_Euler_Cpp) ships its own run outputs under
code_test/, accuracy_test/ and speed_test/.  These files are reference OUTPUT data, not source;
this script copies the small ones that pin the 2D and 1D hot paths so the tests can run where the
reference tree is not mounted.  Run it once in a container that has the reference:

    python tests/golden/make_golden.py [/path/to/reference]
"""
import json
import shutil
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent

# (source path inside the reference, destination name)
FILES = []
# 4x4 k=2 production-path checks (code_test/2d/test_solver.py:13-21), current exact block Jacobi
for case in ("be", "dirk3", "entropy"):
    for part in ("iterations", "summary", "difference"):
        FILES.append((f"code_test/2d/results/exact_only_20261019/{case}_{part}.csv",
                      f"c4x4_{case}_{part}.csv"))
    FILES.append((f"code_test/2d/results/exact_only_20261019/{case}.command.json",
                  f"c4x4_{case}.command.json"))
# The only archived 2D nodal solution: 4x4 k=2 DIRK3 T=0.02
for part in ("solution", "summary", "iterations", "difference"):
    FILES.append((f"code_test/2d/results/first_dirk_{part}.csv", f"first_dirk_{part}.csv"))
# 2D accuracy family, Q2 DIRK3 CFL2 T0.2 (config 64^2 k=2)
ACC = "accuracy_test/results/2d_submission_20261019T234902_AtKkgL/job_7640912/data"
for n in (32, 64, 128, 256):
    FILES.append((f"{ACC}/n{n}_summary.csv", f"acc_n{n}_summary.csv"))
    FILES.append((f"{ACC}/n{n}.command.json", f"acc_n{n}.command.json"))
for n in (32, 64, 128, 256):
    FILES.append((f"{ACC}/n{n}_iterations.csv", f"acc_n{n}_iterations.csv"))
FILES.append((f"{ACC}/convergence.csv", "acc_convergence.csv"))
# 2D speed family, 256^2 BE CFL5 four updates (config 256^2 k=8 and k=0..7)
SPD = "speed_test/results/2d_submission_20261019T205542_KhFC6z/job_7635952/data"
for k in range(9):
    for m in ("dg", "hdg"):
        FILES.append((f"{SPD}/k{k}_{m}_iterations.csv", f"speed256_k{k}_{m}_iterations.csv"))
        FILES.append((f"{SPD}/k{k}_{m}_summary.csv", f"speed256_k{k}_{m}_summary.csv"))
FILES.append((f"{SPD}/k8_dg.command.json", "speed256_k8_dg.command.json"))
# 512^2 k=8, BE CFL5 four updates, GMRES(30) (DG and HDG ran as separate jobs)
N512 = "speed_test/results/2d_n512_restart30_20261020T220633_rt2c3wx6"
for m, job in (("dg", "job_7718103"), ("hdg", "job_7687732")):
    for part in ("iterations", "summary"):
        FILES.append((f"{N512}/{job}/data/k8_{m}_{part}.csv", f"speed512_k8_{m}_{part}.csv"))
    FILES.append((f"{N512}/{job}/data/k8_{m}.command.json", f"speed512_k8_{m}.command.json"))
# 1D production-path checks (code_test/1d/test_solver.py): 32 cells k=3 one BE step and
# 16 cells k=2 DIRK3 to T=0.02, DG and HDG, block-Jacobi GMRES, with their commands
ONE = "code_test/1d/results/intel_final_20261019"
for case in ("be_update", "dirk_smoke"):
    for part in ("iterations", "summary", "solution", "difference"):
        FILES.append((f"{ONE}/{case}_{part}.csv", f"d1_{case}_{part}.csv"))
    FILES.append((f"{ONE}/{case}.command.json", f"d1_{case}.command.json"))
# 1D k=8, 32 cells, one BE step (command not archived; the summary holds its parameters)
for part in ("iterations", "summary", "solution", "difference"):
    FILES.append((f"code_test/1d/results/k8_n32_check_{part}.csv", f"d1_k8_n32_{part}.csv"))
# 1D accuracy family, k=2 DIRK3 CFL2 T0.2, N = 32..512 (config N=64 k=2)
FILES.append(("accuracy_test/results/1d_intel_20261019/convergence_intel_20261019.csv", "d1_convergence.csv"))


def main() -> None:
    ref = Path(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
    manifest = {}
    for src, dst in FILES:
        path = ref / src
        if not path.exists():
            print("missing", src)
            continue
        shutil.copyfile(path, HERE / dst)
        manifest[dst] = src
    (HERE / "MANIFEST.json").write_text(json.dumps(manifest, indent=1, sort_keys=True) + "\n")
    print(f"copied {len(manifest)} files")


if __name__ == "__main__":
    main()
