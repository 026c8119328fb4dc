"""The tool's process chain solved on the GPU, on the reference's own models built by the restated
model-building side (the mesher, the substrate bands, the parts' tables from the database records
of tests/golden/materials_subset.json, the chain's stages with their births). The file runs after
the kernel-level GPU tests: it drives whole analyses.

* The default package at Draft (65,322 DOF, 15 steps 217 -> 165 -> 150 -> 25 degC): every step's
  increment within 1e-8 of the oracle's in FP64 and 1e-5 in mixed precision (both solved to
  relative residual 1e-12; the oracle takes about a minute on one core), and the room-temperature
  JEITA warpage at the reference's published -69.34 um (README.md:91) to its printed digits.
* The bare-die preset (V9, src/core/15-verify.js:339-357; README.md:358): the warpage +222.7 um
  and the die backside interior peak +65.8 MPa from the die's element states marched on the
  device (accumulateStep, stateStress), to their printed digits.
* V10's Standard half (README.md:358): the default package at Standard (314,385 DOF), -69.3 um
  and the die interior peak 72.6 MPa.
* V18's bare module package (15-verify.js:573-636; README.md:366: a Si-base module with two
  chiplets, its module stages free on their three-point support, then the substrate's): the RT
  warpage +11.04 um, the whole-face Gauss-point peaks of the chiplets 49.6 / 5.3 MPa and of the Si
  base 20.2 / 18.3 MPa, the worst DDI microbump shear 75.3 mN and the wafer underfill sidewall shear
  4.43 MPa, to their printed digits."""
import json
import os

import numpy as np
import pytest

from tmsolve import post
from tmsolve.analysis import process_chain, process_package, solve_chain
from tmsolve.pkgmesh import default_config, preset_config

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "materials_subset.json")


def _bga(cfg):
    return post.bga_sites(sx=cfg["substrate"]["sx"], sy=cfg["substrate"]["sy"], inset=cfg["bga"]["inset"], pitch=cfg["bga"]["pitch"])


def test_default_package_chain_on_gpu(oracle_lib):
    from tmsolve.solver import DeviceModel
    recs = json.load(open(GOLDEN))
    cfg = default_config()
    pkg = process_package(cfg, recs, "draft")
    steps = process_chain(pkg, recs)
    b = _bga(cfg)
    z = b["zone"]
    om = oracle_lib.OracleModel(pkg)
    uo, ro, _ = solve_chain(om, pkg, steps, tol=1e-12)
    assert all(r["converged"] for r in ro)
    wo = om.warpage_jeita(uo, b["x"], b["y"], [z["x0"], z["x1"], z["y0"], z["y1"]])["signed"]
    for precision, bar in (("fp64", 1e-8), ("mixed", 1e-5)):
        dm = DeviceModel(pkg)                    # its own stored solutions: the same warm starts as the oracle's
        try:
            u, rs, _ = solve_chain(dm, pkg, steps, tol=1e-12, precision=precision)
            assert all(r["converged"] for r in rs), (precision, [r["relres"] for r in rs])
            for k, (r, o) in enumerate(zip(rs, ro)):
                assert np.linalg.norm(r["u"] - o["u"]) <= bar * np.linalg.norm(o["u"]), (precision, k)
            w = post.warpage_jeita(b, lambda x, y: dm.sample_plane(u, 0, 2, x, y))["signed"]
        finally:
            dm.close()
        assert abs(w / wo - 1) <= bar, (precision, w, wo)
        assert f"{1000 * w:.2f}" == "-69.34", (precision, w)


def _die_rt_on_gpu(cfg, preset):
    """The chain of a single-die configuration solved on the GPU: the signed JEITA warpage (mm) and
    the die's top-face stress record from its element states marched on the device."""
    from tmsolve.mesh import PART
    from tmsolve.solver import DeviceModel
    recs = json.load(open(GOLDEN))
    pkg = process_package(cfg, recs, preset)
    d = pkg.meta["mesh_info"]["geometry"]["dies"][0]
    group = 3                                    # packageGroups: substrate, solder, underfill, then the dies
    kp = post.plane_index(pkg.mesh, d["ztop"])
    elems = np.array([e for (_, _, e) in post.die_elements(pkg.mesh, d["rect"], kp - 1, PART["DIE"], group)[0]], np.int32)
    b = _bga(cfg)
    dm = DeviceModel(pkg)
    try:
        u, rs, S = solve_chain(dm, pkg, process_chain(pkg, recs), state_elems=elems)
        assert all(r["converged"] for r in rs)
        w = post.warpage_jeita(b, lambda x, y: dm.sample_plane(u, 0, 2, x, y))["signed"]
        ds = post.die_surface_stress(dm, S, elems, S.shape[1], d["rect"], d["ztop"], d["zaf"], PART["DIE"], group, "top")
    finally:
        dm.close()
    return w, ds


def test_bare_die_v9_on_gpu():
    w, ds = _die_rt_on_gpu(preset_config("bare"), "draft")
    assert f"{1000 * w:.1f}" == "222.7" and f"{ds['peakInterior']:.1f}" == "65.8", (w, ds["peakInterior"])


def test_default_package_v10_standard_on_gpu():
    """V10's Standard half (15-verify.js; README.md:358: -69.3 um and a die interior peak of
    72.6 MPa at Standard, 314k DOF with 2 layers per region) with the chain on the GPU."""
    w, ds = _die_rt_on_gpu(default_config(), "standard")
    assert f"{1000 * w:.1f}" == "-69.3" and f"{ds['peakInterior']:.1f}" == "72.6", (w, ds["peakInterior"])


def test_v18_module_package_on_gpu():
    from test_host_modules import V18_OPTS, check_v18, v18_config, v18_results
    from tmsolve.solver import DeviceModel
    recs = json.load(open(GOLDEN))
    cfg = v18_config()
    pkg = process_package(cfg, recs, "draft", V18_OPTS)
    dm = DeviceModel(pkg)
    try:
        res = v18_results(dm, pkg, recs, cfg, lambda u, b: post.warpage_jeita(b, lambda x, y: dm.sample_plane(u, 0, 2, x, y)))
    finally:
        dm.close()
    check_v18(res)


def test_v8_symmetry_on_gpu():
    """The reference's check V8 (src/core/15-verify.js:312-337) with the chains solved on the GPU:
    the centred bare die's residual field symmetric in x, y and across the diagonal, and the offset
    die's mirrored with its floorplan, to 1e-6 of the warpage magnitude (the GPU sweeps its columns
    in four colours, so no sweep order favours a side)."""
    from test_host_analysis import v8_symmetry
    from tmsolve.solver import DeviceModel

    def jeita(model, pkg, u):
        return post.warpage_jeita(_bga(pkg.meta["cfg"]), lambda x, y: model.sample_plane(u, 0, 2, x, y))
    rel = v8_symmetry(DeviceModel, jeita)
    assert max(rel) < 1e-6, rel
