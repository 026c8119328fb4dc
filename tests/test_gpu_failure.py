"""Failure detection without a GPU fault, and the solve's progress callback.

Every device wait of the library is bounded. A wait that runs out makes the kernel flag the error,
let its copies in flight land and return; the host reports TM_TIMEOUT and the context stays usable.
The test hook tm_set_wait_test makes the level-0 TMA sweep (used for a caller-assembled operator,
tm_set_bcsr, in mixed precision) wait with a short limit for a stage flag that nothing sets; no
kernel faults, traps or hangs.
"""
import numpy as np
import pytest

from tmsolve import _lib
from tmsolve.materials import iso_d
from tmsolve.packages import box_package, fcbga_c1, linspace

pytestmark = pytest.mark.gpu


def test_bounded_wait_timeout_is_reported_and_context_survives(oracle_lib):
    from tmsolve.solver import DeviceModel
    pkg = fcbga_c1()
    dm = DeviceModel(pkg)
    om = oracle_lib.OracleModel(pkg)
    fo = om.assemble(pkg.step())
    rp, col, val, isC = om.bcsr()
    dm.set_bcsr(rp, col, val, isC)
    dm.set_wait_test(True)
    with pytest.raises(_lib.TmError) as e:
        dm.solve(fo, tol=1e-10, maxit=3, warm=0, key=1, precision="mixed")
    assert e.value.status == _lib.TM_TIMEOUT
    assert "wait" in str(e.value)
    dm.set_wait_test(False)
    r = dm.solve(fo, tol=1e-10, warm=0, key=2, precision="mixed")
    r64 = dm.solve(fo, tol=1e-10, warm=0, key=3)
    assert r["converged"] and r64["converged"]
    assert np.linalg.norm(r["u"] - r64["u"]) / np.linalg.norm(r64["u"]) <= 1e-5


def test_progress_callback():
    """progress(it, relres) between PCG iterations, every progress_every iterations (LIVE.post)."""
    from tmsolve.solver import DeviceModel
    mats = [(iso_d(110000.0, 0.34), 16.4e-6, 16.4e-6), (iso_d(130000.0, 0.28), 2.6e-6, 2.6e-6)]
    pkg = box_package(linspace(-5, 5, 8), linspace(-4, 4, 6), [0, 0.25, 0.5, 0.75, 1.0], mats,
                      lambda i, j, k: 0 if k < 2 else 1, Ta=25.0, Tb=-75.0)
    dm = DeviceModel(pkg)
    calls = []
    r = dm.solve(dm.assemble_step(pkg.step()), tol=1e-12, warm=0, progress=lambda it, rel: calls.append((it, rel)),
                 progress_every=2)
    assert r["converged"] and r["iters"] >= 4
    assert [c[0] for c in calls] == list(range(2, r["iters"] + 1, 2))
    assert all(rel > 0 for _, rel in calls)
    assert calls[0][1] > calls[-1][1]
    if r["iters"] % 2 == 0:
        assert calls[-1][1] == pytest.approx(r["relres"], rel=1e-12)
