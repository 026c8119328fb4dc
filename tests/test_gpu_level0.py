"""The matrix-free level-0 operator (tm_set_level0(ctx, 1)): products cell by cell with the element
classes' matrices instead of the assembled 27-point stencil, in the PCG apply and in the V-cycle's
level-0 residuals and column sweeps.

Bars: the apply within 1e-13 of the oracle's fullMatVec (10-solver.js:15-33: the same operator summed
in another order); one FP64 V-cycle within 1e-11 of the stencil path's on the same residual (the
same smoother and hierarchy, summation order only); solutions at relative residual 1e-12 within
1e-8 of the oracle (FP64) and 1e-5 (mixed precision), iteration counts within a few of the stencil
path's.
"""
import numpy as np
import pytest

from tmsolve.packages import fcbga_c1, lidded_c2, rms_warpage

from test_gpu_parity import small_box

pytestmark = pytest.mark.gpu

CASES = [small_box, fcbga_c1, lambda: lidded_c2(n_inplane=24)]
IDS = ["box", "c1", "c2_24"]


def _mf_model(pkg):
    from tmsolve.solver import DeviceModel
    dm = DeviceModel(pkg)
    dm.set_level0(True)
    return dm


@pytest.mark.parametrize("make", CASES, ids=IDS)
def test_matrix_free_apply_matches_oracle(make, oracle_lib):
    pkg = make()
    dm, om = _mf_model(pkg), oracle_lib.OracleModel(pkg)
    step = pkg.step()
    dm.assemble_step(step); om.assemble(step)
    assert dm.level0_matrix_free
    x = np.random.default_rng(3).standard_normal(dm.ndof)
    y, yo = dm.matvec(x), om.matvec(x)
    assert np.linalg.norm(y - yo) / np.linalg.norm(yo) <= 1e-13


def test_default_is_the_stencil():
    from tmsolve.solver import DeviceModel
    pkg = fcbga_c1()
    dm = DeviceModel(pkg)
    dm.assemble_step(pkg.step())
    assert not dm.level0_matrix_free
    dm.set_level0(True)
    assert not dm.level0_matrix_free          # takes effect at the next assembly
    dm.assemble_step(pkg.step())
    assert dm.level0_matrix_free
    dm.set_level0(False)
    dm.assemble_step(pkg.step())
    assert not dm.level0_matrix_free


@pytest.mark.parametrize("make", CASES, ids=IDS)
def test_matrix_free_vcycle_matches_stencil(make):
    """One FP64 V-cycle (pc.apply) of each path on the same scaled residual."""
    from tmsolve.solver import DeviceModel
    pkg = make()
    step = pkg.step()
    out = []
    for mf in (False, True):
        dm = DeviceModel(pkg)
        dm.set_level0(mf)
        f = dm.assemble_step(step)
        r = dm.solve(f, tol=1e-6, precision="fp64")
        assert r["converged"] and dm.level0_matrix_free == mf
        rr = np.random.default_rng(5).standard_normal(dm.ndof)
        out.append(dm.pc_apply(rr))
    assert np.linalg.norm(out[1] - out[0]) / np.linalg.norm(out[0]) <= 1e-11


@pytest.mark.parametrize("make", [small_box, fcbga_c1, lambda: lidded_c2(n_inplane=48)], ids=["box", "c1", "c2_48"])
@pytest.mark.parametrize("precision, bar", [("fp64", 1e-8), ("mixed", 1e-5)])
def test_matrix_free_solve_matches_oracle(make, precision, bar, oracle_lib):
    from tmsolve.solver import DeviceModel
    pkg = make()
    step = pkg.step()
    om = oracle_lib.OracleModel(pkg)
    ro = om.solve(om.assemble(step), tol=1e-12)
    assert ro["converged"]
    st = DeviceModel(pkg)
    rs = st.solve(st.assemble_step(step), tol=1e-12, precision=precision)
    dm = _mf_model(pkg)
    r = dm.solve(dm.assemble_step(step), tol=1e-12, precision=precision)
    assert r["converged"] and dm.level0_matrix_free
    u, uo = r["u"], ro["u"]
    assert np.linalg.norm(u - uo) / np.linalg.norm(uo) <= bar
    assert abs(rms_warpage(pkg.mesh, u) / rms_warpage(pkg.mesh, uo) - 1) <= bar
    assert abs(r["iters"] - rs["iters"]) <= 3, (r["iters"], rs["iters"])


def test_matrix_free_module_stage():
    """The module step (stage -1: born module parts only, held package) and the first whole-package
    step after it, matrix-free against the stencil path."""
    from tmsolve.packages import module_path_steps, stacked_module
    from tmsolve.solver import DeviceModel
    pkg = stacked_module(24)
    steps = module_path_steps(pkg)[0][:2]
    sols = []
    for mf in (False, True):
        dm = DeviceModel(pkg)
        dm.set_level0(mf)
        us = []
        for k, st in enumerate(steps):
            r = dm.solve(dm.assemble_step(st), tol=1e-12, key=k, precision="fp64")
            assert r["converged"] and dm.level0_matrix_free == mf
            us.append(r["u"])
        sols.append(us)
    for a, b in zip(*sols):
        assert np.linalg.norm(b - a) / np.linalg.norm(a) <= 1e-8
