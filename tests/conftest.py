import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "oracle"))
GOLDEN = Path(__file__).resolve().parent / "golden"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: takes more than a few seconds on CPU")


@pytest.fixture(scope="session")
def oracle_mod():
    import oracle_py

    oracle_py.lib()  # builds the oracle with make when absent
    return oracle_py


def read_csv(path):
    import csv

    with open(path, newline="") as fh:
        return list(csv.DictReader(fh))


def assert_history_close(ours, ref, rtol=1e-10, switch_rel=1e-6, floor_rel=1e-10, krylov_slack=1):
    """Residual histories: relative (rtol) where the value is above switch_rel*r0, and an
    absolute floor of floor_rel*r0 below it, r0 being the largest residual of the run.  Late
    Newton residuals sit at the linear-solve tolerance, where only an absolute bound means
    anything.

    Krylov counts may differ by +-krylov_slack near the tolerance (rounding order differs).
    """
    assert len(ours) == len(ref), (len(ours), len(ref))
    r0 = max(float(r["residual_physical_rms"]) for r in ref)
    for a, b in zip(ours, ref):
        for key in ("method", "step", "stage", "iteration"):
            assert a[key] == b[key], (key, a[key], b[key])
        for key in ("time", "stage_time", "dt", "cfl"):
            assert abs(float(a[key]) - float(b[key])) <= 1e-12 * max(1.0, abs(float(b[key]))), (key, a, b)
        x, y = float(a["residual_physical_rms"]), float(b["residual_physical_rms"])
        if abs(y) > switch_rel * r0:
            assert abs(x - y) <= rtol * abs(y), ("rms", x, y)
        else:
            assert abs(x - y) <= floor_rel * r0, ("rms floor", x, y)
        assert abs(int(a["krylov_iterations"]) - int(b["krylov_iterations"])) <= krylov_slack, (a, b)
