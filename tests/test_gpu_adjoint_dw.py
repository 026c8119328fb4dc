"""Adjoint gradient of a bump's last-cycle dW (the peak bump of a stacked module over three
-40/125 degC cycles) with respect to the property sets' stiffness and thermal strain, against
central finite differences of the whole analysis (every path step re-solved, the strain table
rebuilt, the site re-screened) with a relative step of 1e-4.

The finite differences keep the increments in FP64 (the analysis itself keeps them as float32,
whose rounding would be amplified 1e4 times by the difference quotient); the gradient is taken on
the same path. Bars: the screening's forward-mode dW equals the screening's own to 1e-12, and every
checked component agrees with its difference quotient within 1e-4 of the larger of the two, or
1e-6 of the gradient's largest component where the component itself is that small.
"""
import numpy as np
import pytest

from tmsolve import post
from tmsolve.anand import cycle_history, cycling_temps, screen
from tmsolve.materials import SAC305_MODULE, anand_tables
from tmsolve.packages import module_path_steps, stacked_module
from tmsolve.sensitivity import scale_step, site_dw_gradient

pytestmark = pytest.mark.gpu


def test_peak_bump_dw_gradient_matches_central_differences():
    from tmsolve.solver import DeviceModel
    pkg = stacked_module(24)
    temps = cycling_temps(-40.0, 125.0)
    steps, Tb, chain, up, down = module_path_steps(pkg, temps=temps)
    dm = DeviceModel(pkg)
    bl = pkg.meta["bump_layer"]
    hist = cycle_history(-40.0, 125.0, 11.0, 15.0, 3, ramp_max_dt=10.0, dwell_steps=3)
    Et, Ft = anand_tables(SAC305_MODULE)
    key = [0]

    def solve_path(stp):
        us = []
        for st in stp:
            key[0] += 1
            r = dm.solve(dm.assemble_step(st), tol=1e-12, warm=0, key=key[0])
            assert r["converged"]
            us.append(r["u"])
        return us

    def site_dw(stp, us, x, y):
        tab = post.site_strain_table(dm, post.ThermalPath(stp, Tb, us, chain, up, down), dict(x=np.array([x]), y=np.array([y])), temps,
                                     bl["zmid"], bl["part"])
        return screen(SAC305_MODULE, Et, Ft, temps, tab, hist)[0][0]

    us = solve_path(steps)
    path = post.ThermalPath(steps, Tb, us, chain, up, down)
    sites = post.screening_sites(post.bump_field(**pkg.meta["die"]), 48)["sites"]
    table = post.site_strain_table(dm, path, sites, temps, bl["zmid"], bl["part"])
    dW, _, _ = screen(SAC305_MODULE, Et, Ft, temps, table, hist)
    q = int(np.nanargmax(dW))
    x, y = float(sites["x"][q]), float(sites["y"][q])
    g = site_dw_gradient(dm, path, us, x, y, temps, bl["zmid"], bl["part"], SAC305_MODULE, Et, Ft, hist)
    assert g["dW"] == pytest.approx(dW[q], rel=1e-12)
    scale = max(np.abs(g["dlogE"]).max(), np.abs(g["dlogA"]).max())
    assert scale > 0
    h = 1e-4
    # substrate, bump-layer solder, bump-layer underfill, Si base die: stiffness and thermal strain
    for m, kind in ((0, "E"), (1, "E"), (2, "E"), (3, "E"), (0, "A"), (3, "A")):
        vals = []
        for f in (1 + h, 1 - h):
            stp = [scale_step(st, m, stiffness=f if kind == "E" else 1.0, thermal=f if kind == "A" else 1.0) for st in steps]
            vals.append(site_dw(stp, solve_path(stp), x, y))
        fd = (vals[0] - vals[1]) / (2 * h)
        adj = g["dlogE"][m] if kind == "E" else g["dlogA"][m]
        assert abs(adj - fd) <= max(1e-4 * max(abs(fd), abs(adj)), 1e-6 * scale), (m, kind, adj, fd)
