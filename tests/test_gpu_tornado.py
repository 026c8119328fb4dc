"""The tornado batch (24 perturbed materials of the lidded C2 package in one solve loop, each
warm started from the case before it) against the oracle's fresh solve of every case.

Bars: both sides solved to relative residual 1e-10; the signed JEITA warpage and the RMS warpage of
every case within 1e-7 relative (the warm start changes only the path to the solution)."""
import pytest

from tmsolve import post
from tmsolve.packages import lidded_c2, rms_warpage
from tmsolve.sensitivity import case_scales, tornado, tornado_cases

pytestmark = pytest.mark.gpu


def test_tornado_matches_oracle(oracle_lib):
    from tmsolve.solver import DeviceModel
    pkg = lidded_c2(n_inplane=24)
    dm = DeviceModel(pkg)
    res = tornado(dm, tornado_cases(), tol=1e-10, precision="fp64")
    assert len(res["cases"]) == 24 and len(res["swing"]) == 12
    bga = post.bga_sites(**pkg.meta["bga"])
    z = bga["zone"]
    om = oracle_lib.OracleModel(pkg)
    for q, rec in enumerate([res["base"]] + res["cases"]):
        st = pkg.material_step(case_scales(rec["case"]))
        ro = om.solve(om.assemble(st), tol=1e-10)
        assert ro["converged"]
        wo = om.warpage_jeita(ro["u"], bga["x"], bga["y"], [z["x0"], z["x1"], z["y0"], z["y1"]])
        assert abs(rec["signed"] / wo["signed"] - 1) <= 1e-7, (q, rec["signed"], wo["signed"])
        assert abs(rec["rms"] / rms_warpage(pkg.mesh, ro["u"]) - 1) <= 1e-7, q
    # the cases start from the stored solution of the case before them, which saves iterations
    # against the same loop from zero
    assert all(c["warm"] > 0 for c in res["cases"])
    dm.clear_warm()
    cold = tornado(dm, tornado_cases(), tol=1e-10, precision="fp64", key=1000, warm=0)
    its = lambda r: sum(c["iters"] for c in [r["base"]] + r["cases"])
    assert its(res) < its(cold), (its(res), its(cold))
    for a, b in zip(res["cases"], cold["cases"]):
        assert abs(a["signed"] / b["signed"] - 1) <= 1e-7
    # a stiffer die or a larger expansion mismatch moves the warpage: every input has a swing
    assert all(s["span"] > 0 for s in res["swing"])
