"""The library on the reference's own mesh: the default package (lidded single die) at the Draft
preset, built by the restated ``buildPackageMesh`` (65,322 DOF), solved on the GPU and by the
oracle.

Bars: the assembled load and operator within 1e-13 of the oracle's (same sums, other order of the
slots); solutions at relative residual 1e-12 within 1e-8 of the oracle's in FP64 and 1e-5 in
mixed precision, the RMS warpage likewise; FP64 iterations within 15 % of the oracle's (the GPU
sweeps its columns in four colours, the reference lexicographically)."""
import numpy as np
import pytest

from tmsolve.packages import reference_package, rms_warpage

pytestmark = pytest.mark.gpu


def test_reference_draft_matches_oracle(oracle_lib):
    from tmsolve.solver import DeviceModel
    pkg = reference_package("draft")
    step = pkg.step()
    om = oracle_lib.OracleModel(pkg)
    dm = DeviceModel(pkg)
    # the operators first: a solve scales the oracle's operator in place (_scale)
    fo = om.assemble(step)
    f = dm.assemble_step(step)
    assert np.linalg.norm(f - fo) <= 1e-13 * np.linalg.norm(fo)
    x = np.random.default_rng(11).standard_normal(dm.ndof)
    y, yo = dm.matvec(x), om.matvec(x)
    assert np.linalg.norm(y - yo) <= 1e-13 * np.linalg.norm(yo)
    ro = om.solve(fo, tol=1e-12)
    assert ro["converged"]
    for precision, bar in (("fp64", 1e-8), ("mixed", 1e-5)):
        r = dm.solve(f, tol=1e-12, precision=precision, key=1 if precision == "fp64" else 2)
        assert r["converged"], (precision, r["relres"])
        u, uo = r["u"], ro["u"]
        assert np.linalg.norm(u - uo) <= bar * np.linalg.norm(uo), precision
        assert abs(rms_warpage(pkg.mesh, u) / rms_warpage(pkg.mesh, uo) - 1) <= bar, precision
        if precision == "fp64":
            assert abs(r["iters"] - ro["iters"]) <= max(3, 0.15 * ro["iters"]), (r["iters"], ro["iters"])
