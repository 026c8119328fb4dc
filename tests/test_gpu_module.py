"""The stacked-module thermal-cycle analysis on the GPU against the oracle: the module step (stage
-1), the whole package down to 25 degC and the two cycling branches (module_path_steps), the
bump-layer strain table at the die bump sites from those increments (siteStrainTable), and the
Anand screening of the sites over three -40/125 degC cycles at 40 load steps per cycle with the
module's SAC305 constants.

Bars, stage by stage on identical inputs: every step's displacement increment within 1e-8 (relres
1e-12 on both sides); from the same float32 increments the GPU and the oracle build the same
strain table to 1e-12 of its largest entry; from the same table they screen the same dW and dE to
1e-8 per site. End to end, each side from its own increments: the analysis keeps the increments as
float32 (11-analysis.js:256), so increments that agree to 1e-8 can round to neighbouring floats and
the tables differ by up to a few float32 ulps (bar 1e-6 of the largest entry). The screening is a
hysteresis-energy difference of nearly cancelling strain excursions, which amplifies that
difference at the sites with the smallest dW: the end-to-end bar is 1e-5 relative on the median
site and 1e-3 on every site, the largest measured error printed.
"""
import numpy as np
import pytest

from tmsolve import post
from tmsolve.anand import cycle_history, cycling_temps, screen
from tmsolve.materials import SAC305_MODULE, anand_params_array, anand_tables
from tmsolve.packages import module_path_steps, stacked_module

pytestmark = pytest.mark.gpu


def test_module_thermal_cycle_matches_oracle(oracle_lib):
    from tmsolve.solver import DeviceModel
    pkg = stacked_module(32)
    steps, Tb, chain, up, down = module_path_steps(pkg)
    dm, om = DeviceModel(pkg), oracle_lib.OracleModel(pkg)
    dg, do = [], []
    for k, st in enumerate(steps):
        r = dm.solve(dm.assemble_step(st), tol=1e-12, key=k)
        ro = om.solve(om.assemble(st), tol=1e-12, key=k)
        assert r["converged"] and ro["converged"], k
        assert np.linalg.norm(r["u"] - ro["u"]) <= 1e-8 * np.linalg.norm(ro["u"]), k
        dg.append(r["u"].astype(np.float32).astype(np.float64))
        do.append(ro["u"].astype(np.float32).astype(np.float64))
    sites = post.screening_sites(post.bump_field(**pkg.meta["die"]), 400)["sites"]
    temps = cycling_temps(-40.0, 125.0)
    bl = pkg.meta["bump_layer"]
    tg = post.site_strain_table(dm, post.ThermalPath(steps, Tb, dg, chain, up, down), sites, temps, bl["zmid"], bl["part"])
    to = post.site_strain_table(om, post.ThermalPath(steps, Tb, do, chain, up, down), sites, temps, bl["zmid"], bl["part"])
    ok = np.isfinite(to)
    assert ok.mean() > 0.9 and np.array_equal(ok, np.isfinite(tg))
    assert np.abs(tg[ok] - to[ok]).max() <= 1e-6 * np.abs(to[ok]).max()
    tgo = post.site_strain_table(om, post.ThermalPath(steps, Tb, dg, chain, up, down), sites, temps, bl["zmid"], bl["part"])
    assert np.abs(tg[ok] - tgo[ok]).max() <= 1e-12 * np.abs(tgo[ok]).max()
    hist = cycle_history(-40.0, 125.0, 11.0, 15.0, 3, ramp_max_dt=10.0, dwell_steps=3)
    Et, Ft = anand_tables(SAC305_MODULE)
    oW, oE, _ = oracle_lib.anand_screen(anand_params_array(SAC305_MODULE), Et, Ft, temps, to, hist)
    fin = np.isfinite(oW)
    assert fin.mean() > 0.9 and np.all(oW[fin] > 0)
    sW, sE, _ = screen(SAC305_MODULE, Et, Ft, temps, to, hist)           # the oracle's own table
    assert np.array_equal(fin, np.isfinite(sW))
    assert np.allclose(sW[fin], oW[fin], rtol=1e-8, atol=0)
    assert np.allclose(sE[fin], oE[fin], rtol=1e-8, atol=0)
    dW, dE, _ = screen(SAC305_MODULE, Et, Ft, temps, tg, hist)           # end to end
    assert np.array_equal(fin, np.isfinite(dW))
    for a, b, name in ((dW, oW, "dW"), (dE, oE, "dE")):
        rel = np.abs(a[fin] - b[fin]) / np.abs(b[fin])
        print(f"{name}: end-to-end relative error median {np.median(rel):.2e} max {rel.max():.2e}")
        assert np.median(rel) <= 1e-5 and rel.max() <= 1e-3
