"""IC(0) on the GPU (ICPC, src/core/10-solver.js:719-800) and the solve policy's fallback
(:967-976) against the oracle.

Bars: the IC(0) factor of the scaled operator and its apply are bit-exact (every row gathers its
updates in the reference's row order, without fused multiply-add), so pc.apply(r) returns the
oracle's doubles; IC(0)-PCG solutions at relres 1e-12 agree to 1e-8 (the PCG dots sum in a
different order, so iteration counts may differ by a few).
"""
import numpy as np
import pytest

from tmsolve import _lib
from tmsolve.materials import iso_d
from tmsolve.packages import box_package, fcbga_c1, linspace

pytestmark = pytest.mark.gpu


def small_box():
    mats = [(iso_d(110000.0, 0.34), 16.4e-6, 16.4e-6), (iso_d(130000.0, 0.28), 2.6e-6, 2.6e-6)]
    return box_package(linspace(-5, 5, 8), linspace(-4, 4, 6), [0, 0.25, 0.5, 0.75, 1.0], mats,
                       lambda i, j, k: 0 if k < 2 else 1, Ta=25.0, Tb=-75.0)


@pytest.mark.parametrize("make", [small_box, fcbga_c1], ids=["box", "c1"])
def test_ic_apply_bit_exact_and_solve(make, oracle_lib):
    from tmsolve.solver import DeviceModel
    pkg = make()
    dm, om = DeviceModel(pkg), oracle_lib.OracleModel(pkg)
    step = pkg.step()
    f = dm.assemble_step(step)
    fo = om.assemble(step)
    assert np.array_equal(f, fo)
    r = dm.solve(f, tol=1e-12, precond="ic", maxit=20000, warm=0)
    ro = om.solve(fo, tol=1e-12, precond="ic", maxit=20000)
    assert r["converged"] and ro["converged"] and r["precond"] == "ic"
    u, uo = r["u"], ro["u"]
    assert np.linalg.norm(u - uo) / np.linalg.norm(uo) <= 1e-8
    assert abs(r["iters"] - ro["iters"]) <= max(3, 0.05 * ro["iters"])
    x = np.random.default_rng(5).standard_normal(dm.ndof)
    z, zo = dm.pc_apply(x), om.pc_apply(x)
    assert np.array_equal(z, zo), np.abs(z - zo).max()


def test_fallback_to_ic_and_back(oracle_lib):
    """A multigrid run that fails after a fresh build falls back once to IC(0) from the current
    iterate; the next solve uses multigrid again (needRebuild)."""
    from tmsolve.solver import DeviceModel
    pkg = small_box()
    dm, om = DeviceModel(pkg), oracle_lib.OracleModel(pkg)
    step = pkg.step()
    f = dm.assemble_step(step)
    fo = om.assemble(step)
    r = dm.solve(f, tol=1e-10, maxit=2, warm=0)
    ro = om.solve(fo, tol=1e-10, maxit=2)
    assert not r["converged"] and not ro["converged"]
    assert r["fallback"] == dict(first="mg", iters=2, relres=pytest.approx(r["fallback"]["relres"]))
    assert r["precond"] == "ic" and ro["precond"] == "ic" and ro["fallback"] == 1
    assert r["iters"] == ro["iters"] == 4
    dm.assemble_step(step); om.assemble(step)
    r2 = dm.solve(f, tol=1e-10, warm=0)
    assert r2["converged"] and r2["precond"] == "mg" and r2["rebuilt"] and r2["fallback"] is None


def test_pc_apply_needs_a_solve():
    from tmsolve.solver import DeviceModel
    dm = DeviceModel(small_box())
    dm.assemble_step(small_box().step())
    with pytest.raises(_lib.TmError):
        dm.pc_apply(np.zeros(dm.ndof))
