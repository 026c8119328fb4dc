"""The library on the reference's own mesh: the default package (lidded single die) at the Draft
preset, built by the restated ``buildPackageMesh`` (65,322 DOF), solved on the GPU and by the
oracle.

Bars: the assembled operator within 1e-13 of the oracle's (same sums, other order of the slots);
solutions at relative residual 1e-10 within 1e-8 of the oracle's in FP64 and 1e-5 in mixed
precision, the RMS warpage likewise; FP64 iterations within 3 of the oracle's."""
import numpy as np
import pytest

from tmsolve.packages import reference_package, rms_warpage

pytestmark = pytest.mark.gpu


def test_reference_draft_matches_oracle(oracle_lib):
    from tmsolve.solver import DeviceModel
    pkg = reference_package("draft")
    step = pkg.step()
    om = oracle_lib.OracleModel(pkg)
    fo = om.assemble(step)
    ro = om.solve(fo, tol=1e-10)
    assert ro["converged"]
    dm = DeviceModel(pkg)
    f = dm.assemble_step(step)
    assert np.linalg.norm(f - fo) <= 1e-13 * np.linalg.norm(fo)
    x = np.random.default_rng(11).standard_normal(dm.ndof)
    y, yo = dm.matvec(x), om.matvec(x)
    assert np.linalg.norm(y - yo) <= 1e-13 * np.linalg.norm(yo)
    for precision, bar in (("fp64", 1e-8), ("mixed", 1e-5)):
        r = dm.solve(f, tol=1e-10, precision=precision, key=1 if precision == "fp64" else 2)
        assert r["converged"], (precision, r["relres"])
        u, uo = r["u"], ro["u"]
        assert np.linalg.norm(u - uo) <= bar * np.linalg.norm(uo), precision
        assert abs(rms_warpage(pkg.mesh, u) / rms_warpage(pkg.mesh, uo) - 1) <= bar, precision
        if precision == "fp64":
            assert abs(r["iters"] - ro["iters"]) <= 3, (r["iters"], ro["iters"])
