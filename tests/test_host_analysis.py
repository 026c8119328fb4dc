"""The tool's process chain on its default package, on the host and the oracle, against the
reference's published whole-package result: the as-assembled warpage at room temperature of
the default lidded single die at the Draft preset, -69.34 um (README.md:91, the per-preset layers
of PR 40; the JEITA signed warpage at 25 degC after the chain 217 -> 165 degC (S1: die and
solder), 165 -> 150 (S2: underfill), 150 -> 25 (S3: lid, TIM, adhesive)).

Everything on the path is the restated model-building side: the mesh (``pkgmesh``), the
substrate bands and the parts' tables from the database records of the default package's
materials (tests/golden/materials_subset.json, extracted by make_material_fixtures.py), the
thermal path with its births, solved step by step by the oracle."""
import json
import os

import numpy as np

from tmsolve import post
from tmsolve.analysis import process_chain, process_package, solve_chain
from tmsolve.pkgmesh import default_config

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "materials_subset.json")


def test_default_package_chain_steps():
    recs = json.load(open(GOLDEN))
    pkg = process_package(default_config(), recs, "draft")
    steps = process_chain(pkg, recs)
    # S1 with the substrate's Tg (abf_gl 153 and 171 degC) within reach, S2 with the underfill's
    # (111, 112), S3 down to 25 degC; the last step is V11's "S3 30 to 25 degC"
    assert steps[:4] == [(217.0, 187.0, 1), (187.0, 177.0, 1), (177.0, 167.0, 1), (167.0, 165.0, 1)]
    assert steps[4:6] == [(165.0, 155.0, 2), (155.0, 150.0, 2)]
    assert steps[-1] == (30.0, 25.0, 3) and len(steps) == 15
    assert pkg.mesh.ndof == 65322


def test_default_package_rt_warpage(oracle_lib):
    recs = json.load(open(GOLDEN))
    cfg = default_config()
    pkg = process_package(cfg, recs, "draft")
    om = oracle_lib.OracleModel(pkg)
    u, rs, _ = solve_chain(om, pkg, process_chain(pkg, recs))
    assert all(r["converged"] for r in rs)
    b = post.bga_sites(sx=cfg["substrate"]["sx"], sy=cfg["substrate"]["sy"], inset=cfg["bga"]["inset"], pitch=cfg["bga"]["pitch"])
    z = b["zone"]
    w = om.warpage_jeita(u, b["x"], b["y"], [z["x0"], z["x1"], z["y0"], z["y1"]])
    assert f"{1000 * w['signed']:.2f}" == "-69.34", w["signed"]


def _rt(oracle_lib, cfg, recs, die_stress=False):
    """The as-assembled 25 degC state of a configuration at Draft on the oracle: the signed JEITA
    warpage (mm) and, with die_stress, the first die's backside (top face) stress reader."""
    from tmsolve.mesh import PART
    pkg = process_package(cfg, recs, "draft")
    om = oracle_lib.OracleModel(pkg)
    elems, d, group = None, None, None
    if die_stress:
        d = pkg.meta["mesh_info"]["geometry"]["dies"][0]
        group = 3                                # packageGroups: substrate, solder, underfill, then the dies
        kp = post.plane_index(pkg.mesh, d["ztop"])
        elems = np.array([e for (_, _, e) in post.die_elements(pkg.mesh, d["rect"], kp - 1, PART["DIE"], group)[0]], np.int32)
    u, rs, S = solve_chain(om, pkg, process_chain(pkg, recs), state_elems=elems)
    assert all(r["converged"] for r in rs)
    b = post.bga_sites(sx=cfg["substrate"]["sx"], sy=cfg["substrate"]["sy"], inset=cfg["bga"]["inset"], pitch=cfg["bga"]["pitch"])
    z = b["zone"]
    w = om.warpage_jeita(u, b["x"], b["y"], [z["x0"], z["x1"], z["y0"], z["y1"]])["signed"]
    ds = None
    if die_stress:
        ds = post.die_surface_stress(om, S, elems, S.shape[1], d["rect"], d["ztop"], d["zaf"], PART["DIE"], group, "top")
    return w, ds


def test_v9_presets(oracle_lib):
    """The reference's check V9 (src/core/15-verify.js:339-357) at Draft, its published values
    (README.md:358: "bare RT +222.7 um convex; backside +65.8 MPa tensile; 0.8 mm core 166.0 vs
    285.8 um; 795G LH 169.5 vs 705G 263.6 um") to their printed digits: the bare-die preset's
    room-temperature warpage and die backside interior peak stress, the core-thickness study's
    two variants, and the bare package with the 705G and the 795G Type LH cores."""
    from tmsolve.pkgmesh import preset_config
    recs = json.load(open(GOLDEN))
    w, ds = _rt(oracle_lib, preset_config("bare"), recs, die_stress=True)
    assert f"{1000 * w:.1f}" == "222.7" and f"{ds['peakInterior']:.1f}" == "65.8", (w, ds["peakInterior"])
    wa, _ = _rt(oracle_lib, preset_config("coreStudy", "A"), recs)
    wb, _ = _rt(oracle_lib, preset_config("coreStudy", "B"), recs)
    assert f"{1000 * wa:.1f}" == "285.8" and f"{1000 * wb:.1f}" == "166.0", (wa, wb)
    cores = {}
    for core in ("mcl_e_705g", "mcl_e_795g_lh"):
        cfg = preset_config("bare")
        for r in cfg["substrate"]["layers"]:
            if r["type"] == "core":
                r["mat"] = core
        cores[core], _ = _rt(oracle_lib, cfg, recs)
    assert f"{1000 * cores['mcl_e_705g']:.1f}" == "263.6" and f"{1000 * cores['mcl_e_795g_lh']:.1f}" == "169.5", cores


def test_default_package_full_path():
    """A full analysis of the default package solves one step per piece of its thermal path: 67
    steps (README.md:370), the chain (15), the chip-join branch T_UF -> 25 degC in S1, and the sweeps
    from 25 degC down to -40 and up to the 260 degC reflow peak through every evaluation
    temperature (the cycling samples every 10 degC, 5 near a Tg; the reflow sweep; the solidus)."""
    from tmsolve.analysis import full_path
    recs = json.load(open(GOLDEN))
    fp = full_path(process_package(default_config(), recs, "draft"), recs)
    assert len(fp["steps"]) == 67
    assert len(fp["chain"]) == 15 and len(fp["cpi"]) == 10
    t = fp["temps"]
    assert t["all"][0] == -40.0 and t["all"][-1] == 260.0 and 217.0 in t["all"] and 218.0 in t["all"]
    assert fp["steps"][fp["down"][-1]][1] == -40.0 and fp["steps"][fp["up"][-1]][1] == 260.0
    # every evaluation temperature is the end of a sweep step
    ends = {fp["steps"][k][1] for k in fp["down"] + fp["up"]}
    assert set(t["all"]) - {25.0} <= ends


def test_v11_solver_integrity(oracle_lib):
    """The reference's check V11 (src/core/15-verify.js:368-393; README.md:360: "residual 7.5e-11
    (20 iterations), reactions 2.3e-10 of the force scale, energy balance 5.7e-14"): the default
    package's chain at Draft with the solver at 1e-10, each step keyed by its index (so that it
    warm-starts from the stored solutions of the steps before it). The last step (S3 30 -> 25 degC)
    takes the published 20 iterations to the published residual; a re-solve from the stored
    solution, against the unconstrained operator and load, leaves the published reactions at the
    supports; the energy balance is at rounding level (the published 5.7e-14 is one rounding)."""
    recs = json.load(open(GOLDEN))
    pkg = process_package(default_config(), recs, "draft")
    om = oracle_lib.OracleModel(pkg)
    steps = process_chain(pkg, recs)
    _, rs, _ = solve_chain(om, pkg, steps, tol=1e-10)
    last = rs[-1]
    assert steps[-1] == (30.0, 25.0, 3)
    assert last["iters"] == 20 and f"{last['relres']:.1e}" == "7.5e-11", (last["iters"], last["relres"])
    a, b, st = steps[-1]
    step = pkg.step(a, b, stage=st)
    u = om.solve(om.assemble(step), tol=1e-10, key=len(steps) - 1)["u"]
    f = om.assemble(step, no_constraints=True)
    Ku = om.matvec(u)
    fscale = max(np.abs(Ku).max(), np.abs(f).max())
    con = pkg.mesh.constraints
    reac = np.abs(Ku[con] - f[con]).max() / fscale
    assert f"{reac:.1e}" == "2.3e-10", reac
    assert abs(u @ Ku - f @ u) / abs(f @ u) < 1e-12


def v8_symmetry(make_model, jeita, tol=1e-12):
    """The reference's check V8 (src/core/15-verify.js:312-337) through a model: the bare preset's
    room-temperature bottom-surface z field at the mesh nodes less the balls' best-fit plane (the
    JEITA record's residual grid, 12-post.js:95-97; the chain at Draft, solved to tol) against
    itself mirrored left to right, top to bottom and across the diagonal, and the offset
    preset's against that of its floorplan mirrored in x, each relative to the JEITA warpage
    magnitude. make_model(pkg) gives a model, jeita(model, pkg, u) its warpage record."""
    from tmsolve.pkgmesh import preset_config
    recs = json.load(open(GOLDEN))

    def run(cfg):
        pkg = process_package(cfg, recs, "draft")
        model = make_model(pkg)
        try:
            u, rs, _ = solve_chain(model, pkg, process_chain(pkg, recs), tol=tol)
            assert all(r["converged"] for r in rs)
            w = jeita(model, pkg, u)
        finally:
            getattr(model, "close", lambda: None)()
        m = pkg.mesh
        ids = np.asarray(m.nodeId).reshape(m.nx, m.ny, m.nz)[:, :, 0]
        c0, c1, c2 = (float(v) for v in w["plane"])
        grid = u[3 * ids + 2] - (c0 + c1 * np.asarray(m.xs)[:, None] + c2 * np.asarray(m.ys)[None, :])
        return grid, w["mag"]

    g, mag = run(preset_config("bare"))
    ex, ey = np.abs(g - g[::-1, :]).max(), np.abs(g - g[:, ::-1]).max()
    ed = np.abs(g - g.T).max() if g.shape[0] == g.shape[1] else 0.0
    c2 = preset_config("offset")
    c2["dies"][0]["x"] = -c2["dies"][0]["x"]
    g1, mag1 = run(preset_config("offset"))
    g2, _ = run(c2)
    return ex / mag, ey / mag, ed / mag, np.abs(g1 - g2[::-1, :]).max() / mag1


def oracle_jeita(model, pkg, u):
    cfg = pkg.meta["cfg"]
    b = post.bga_sites(sx=cfg["substrate"]["sx"], sy=cfg["substrate"]["sy"], inset=cfg["bga"]["inset"], pitch=cfg["bga"]["pitch"])
    z = b["zone"]
    return model.warpage_jeita(u, b["x"], b["y"], [z["x0"], z["x1"], z["y0"], z["y1"]])


def test_v8_symmetry(oracle_lib):
    """V8 on the oracle: symmetric and mirrored to 1e-6 of the warpage magnitude, the reference's
    criterion (its published figures, 1.5e-11 to 9.8e-13, are rounding-level)."""
    rel = v8_symmetry(oracle_lib.OracleModel, oracle_jeita)
    assert max(rel) < 1e-6, rel
