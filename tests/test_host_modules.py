"""Stacked modules through the restated model-building side, on the oracle, against the reference's
check V18 (src/core/15-verify.js:573-636; README.md:366): a 14 x 14 mm bare package carrying one
7 x 6 mm Si-base module with two 3 x 5 mm chiplets, at Draft under a 20k DOF cap.

Published values pinned here to their printed digits: the uniform-CTE module (every module
material given silicon's CTE) left stressed at 3.87e-5 of E alpha dT after its process stages;
the module support's reactions on the first module step at 6.95e-11 of the force scale; the RT
warpage of the bare module package, +11.04 um convex; the whole-face Gauss-point peaks of the
chiplets (top / bottom) 49.6 / 5.3 MPa and of the Si base 20.2 / 18.3 MPa; the worst DDI microbump
shear 75.3 mN and the wafer underfill sidewall shear 4.43 MPa."""
import copy
import json
import os

import numpy as np

from tmsolve import post
from tmsolve import pkgmesh as pm
from tmsolve.analysis import full_path, process_chain, process_package, solve_chain
from tmsolve.mesh import PART

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "materials_subset.json")


def v18_config():
    """V18's small module package (15-verify.js:577-585)."""
    cfg = pm.preset_config("bare")
    cfg["substrate"]["sx"] = cfg["substrate"]["sy"] = 14
    m = pm.default_module("M1", 0, 0)
    m.update(sx=7, sy=6)
    m["chiplets"] = [pm.default_chiplet("C1", -1.75, 0, 3.0, 5.0), pm.default_chiplet("C2", 1.75, 0, 3.0, 5.0)]
    cfg["dies"] = []
    cfg["modules"] = [m]
    return cfg


V18_OPTS = {"cap": 20000}


def test_v18_mesh_and_path():
    """The module's parts, planes, groups and three-point support; the chain's module stages
    (chiplet join 221 -> 150 degC at the DDI solder's solidus stop, the wafer underfill cure up
    to 180, the wafer mold cure up to the substrate's 217) before the substrate's."""
    recs = json.load(open(GOLDEN))
    pkg = process_package(v18_config(), recs, "draft", V18_OPTS)
    info = pkg.meta["mesh_info"]
    assert not info["scaled"] and info["hmin"] == 0.6 and info["hminLimit"] == 3.0     # the cap allows h_min 0.6 mm
    assert info["nDof"] < 20000
    assert info["groups"][3:] == ["Module 1 / Chiplet 1", "Module 1 / Chiplet 2", "Module 1 Si base", "Module 1 TSV Cu",
                                  "DDI microbumps", "Wafer underfill", "Wafer mold"]
    assert list(pkg.group_stage) == [0, 1, 2, -3, -3, -3, -3, -3, -2, -1]
    assert {"Module 1 base top", "Module 1 chiplet bottom", "Module 1 wCUF fillet top", "Module 1 top"} <= set(info["planeLabels"])
    m = pkg.mesh
    for part in ("CHIPLET", "BASE_SI", "TSV", "DDI_SOLDER", "DDI_FILL", "WCUF_FILLET", "MOLD"):
        assert (m.ePart == PART[part]).any(), part
    mc = m.moduleConstraints
    assert len(mc) == 6 and len(set(mc // 3)) == 3
    kb = int(np.argmin(np.abs(m.zs - info["geometry"]["zaf"])))     # the support nodes are on the base bottom
    on_kb = {int(v) for v in np.asarray(m.nodeId).reshape(m.nx, m.ny, m.nz)[:, :, kb].ravel() if v >= 0}
    assert {int(d) // 3 for d in mc} <= on_kb
    steps = process_chain(pkg, recs)
    assert steps[:4] == [(221.0, 217.0, -3), (217.0, 187.0, -3), (187.0, 157.0, -3), (157.0, 150.0, -3)]
    assert steps[4] == (150.0, 180.0, -2) and steps[5:8] == [(180.0, 190.0, -1), (190.0, 200.0, -1), (200.0, 217.0, -1)]
    assert steps[8][2] == 1 and steps[-1] == (55.0, 25.0, 2) and len(steps) == 24
    fp = full_path(pkg, recs)
    # a full analysis adds the 'ddi' branch: the joined module cooled from the wafer underfill's cure to 25 degC
    assert fp["ddiJoin"] == [0, 1, 2, 3] and fp["steps"][fp["ddi"][-1]][1:3] == (25.0, -3)
    assert fp["chain"][:4] == [0, 1, 2, 3] and len(fp["chain"]) == 24


def test_v18_module_stages():
    """V18 (1): every module material with silicon's CTE, the module stages leave 3.87e-5 of E alpha
    dT in the module parts (stress at each element centre after the module steps, the increments
    used as solved); V18 (2): the three-point support carries 6.95e-11 of the force scale on the
    first module step solved to 1e-10."""
    from oracle import oracle
    oracle.build()
    recs = json.load(open(GOLDEN))
    cfg = v18_config()
    pkg = process_package(cfg, recs, "draft", V18_OPTS)
    om = oracle.OracleModel(pkg)
    a, b, st = process_chain(pkg, recs)[0]
    step = pkg.step(a, b, stage=st)
    u = om.solve(om.assemble(step), tol=1e-10, key=0)["u"]
    f = om.assemble(step, no_constraints=True)
    Ku = om.matvec(u)
    fscale = max(np.abs(Ku).max(), np.abs(f).max())
    mc = pkg.mesh.moduleConstraints
    assert f"{np.abs(Ku[mc] - f[mc]).max() / fscale:.2e}" == "6.95e-11"

    ru = copy.deepcopy(recs)
    for mid in (cfg["stack"]["moldMat"], cfg["stack"]["wcuf"]["mat"], cfg["stack"]["ddi"]["solder"], "cu"):
        ru[mid]["cte"] = copy.deepcopy(ru["si"]["cte"])
        ru[mid].pop("cteXY", None)
        ru[mid].pop("cteZ", None)
    pu = process_package(cfg, ru, "draft", V18_OPTS)
    mod = [s for s in process_chain(pu, ru) if s[2] < 0]
    parts = [PART[k] for k in ("CHIPLET", "BASE_SI", "TSV", "DDI_SOLDER", "DDI_FILL", "WCUF_FILLET", "MOLD")]
    elems = np.array([e for e in range(pu.mesh.ne) if int(pu.mesh.ePart[e]) in parts], np.int32)
    ou = oracle.OracleModel(pu)
    _, rs, S = solve_chain(ou, pu, mod, state_elems=elems, state_f32=False)
    assert len(mod) == 7 and all(r["converged"] for r in rs)
    _, sig = ou.state_stress(elems, S, S.shape[1], np.zeros((len(elems), 3)))
    p = cfg["stack"]["process"]
    scale = 130000 * 3e-6 * max(abs(p["Tddi"] - p["Twcuf"]), abs(p["Tmold"] - cfg["process"]["Tsub"]), 1)
    assert f"{np.abs(sig).max() / scale:.2e}" == "3.87e-05"


def v18_silicon_parts(pkg):
    """(name, rect, ztop, zb, part, group) of the module's silicon parts: the chiplets, the Si base."""
    g = pkg.meta["mesh_info"]["geometry"]
    names = pkg.meta["mesh_info"]["groups"]
    m = g["modules"][0]
    out = [(c["name"], c["rect"], c["ztop"], c["zb"], PART["CHIPLET"], names.index(c["name"])) for c in m["chiplets"]]
    out.append((m["name"] + " Si base", m["rect"], m["zBaseTop"], g["zaf"], PART["BASE_SI"], names.index(m["name"] + " Si base")))
    return out


def v18_state_elements(pkg):
    """The elements that the readers need: the top and bottom element layers of every silicon part,
    the chiplets' microbump-phase elements and the elements around their perimeters."""
    g = pkg.meta["mesh_info"]["geometry"]
    m = g["modules"][0]
    sel = set()
    for (_, rect, zt, zb, part, grp) in v18_silicon_parts(pkg):
        for k in (post.plane_index(pkg.mesh, zt) - 1, post.plane_index(pkg.mesh, zb)):
            sel |= {e for (_, _, e) in post.die_elements(pkg.mesh, rect, k, part, grp)[0]}
    for ci, c in enumerate(m["chiplets"]):
        sel |= set(post.ddi_elements(pkg.mesh, g, 0, ci).tolist())
        sel |= set(post.perimeter_elements(pkg.mesh, c["rect"], m["zDdiTop"], [PART["WCUF_FILLET"], PART["MOLD"]],
                                           PART["DDI_FILL"]).tolist())
    return np.array(sorted(sel), np.int32)


def v18_results(model, pkg, recs, cfg, sampler):
    """The bare module package's 25 degC state through the model: the JEITA warpage, the
    whole-face Gauss-point peaks (top, bottom) of each silicon part, and per chiplet the worst
    microbump shear force (N) and the largest wafer underfill sidewall shear traction (MPa)."""
    g = pkg.meta["mesh_info"]["geometry"]
    elems = v18_state_elements(pkg)
    u, rs, S = solve_chain(model, pkg, process_chain(pkg, recs), state_elems=elems)
    assert all(r["converged"] for r in rs)
    b = post.bga_sites(sx=cfg["substrate"]["sx"], sy=cfg["substrate"]["sy"], inset=cfg["bga"]["inset"], pitch=cfg["bga"]["pitch"])
    w = sampler(u, b)
    st = (S, elems, S.shape[1])
    peaks = {nm: tuple(post.die_surface_stress(model, *st, rect, zt, zb, part, grp, which)["gpPeakAll"] for which in ("top", "bottom"))
             for (nm, rect, zt, zb, part, grp) in v18_silicon_parts(pkg)}
    ddi = [post.ddi_loads(model, *st, g, 0, ci)["worstV"] for ci in range(2)]
    wct = [post.wcuf_tractions(model, *st, g, 0, ci)["maxShearSide"] for ci in range(2)]
    return dict(w=w, peaks=peaks, ddiV=ddi, wcufShear=wct)


def check_v18(res):
    """V18's published 25 degC values (README.md:366) to their printed digits."""
    w, peaks = res["w"], res["peaks"]
    assert w["sign"] > 0 and f"{1000 * w['signed']:.2f}" == "11.04", w["signed"]
    fmt = lambda tb: tuple(f"{v:.1f}" for v in tb)
    assert fmt(peaks["Module 1 / Chiplet 1"]) == ("49.6", "5.3") and fmt(peaks["Module 1 / Chiplet 2"]) == ("49.6", "5.3"), peaks
    assert fmt(peaks["Module 1 Si base"]) == ("20.2", "18.3"), peaks
    assert [f"{1000 * v:.1f}" for v in res["ddiV"]] == ["75.3", "75.3"], res["ddiV"]
    assert [f"{v:.2f}" for v in res["wcufShear"]] == ["4.43", "4.43"], res["wcufShear"]


def test_v18_bare_module_package(oracle_lib):
    """V18 (3): the whole path of the bare module package at 25 degC: warpage, silicon stresses,
    DDI microbump loads (ddiLoads) and wafer underfill tractions (wcufTractions)."""
    recs = json.load(open(GOLDEN))
    cfg = v18_config()
    pkg = process_package(cfg, recs, "draft", V18_OPTS)
    om = oracle_lib.OracleModel(pkg)

    def jeita(u, b):
        z = b["zone"]
        return om.warpage_jeita(u, b["x"], b["y"], [z["x0"], z["x1"], z["y0"], z["y1"]])
    check_v18(v18_results(om, pkg, recs, cfg, jeita))


def test_foveros_preset_meshes():
    """The reference's Foveros-S-like preset (02-config.js:200-208: a 21 x 16 mm Si base die 0.150 mm
    thick with three chiplets, lidded) meshes with every module part under the lid and the
    module's support; its Draft size is a regression value of this restatement (the reference
    publishes only a Fine size, 1.16M DOF, quoted beside a timing run, README.md:420; this mesher
    gives 1,147,032 there)."""
    recs = json.load(open(GOLDEN))
    pkg = process_package(pm.preset_config("foveros"), recs, "draft")
    info = pkg.meta["mesh_info"]
    assert info["nDof"] == 77544 and info["ringRefined"]
    assert info["groups"][6:] == ["Base die 1 / Chiplet 1", "Base die 1 / Chiplet 2", "Base die 1 / Chiplet 3", "Base die 1 Si base",
                                  "Base die 1 TSV Cu", "DDI microbumps", "Wafer underfill", "Wafer mold"]
    for part in ("CHIPLET", "BASE_SI", "TSV", "DDI_SOLDER", "WCUF_FILLET", "MOLD", "TIM", "LID", "LIDADH"):
        assert (pkg.mesh.ePart == PART[part]).any(), part
    assert len(pkg.mesh.moduleConstraints) == 6
    steps = process_chain(pkg, recs)
    assert [s[2] for s in steps[:8]] == [-3, -3, -3, -3, -2, -1, -1, -1] and steps[-1] == (30.0, 25.0, 3)


def test_v18_series_column(oracle_lib):
    """V18 (4): a free-standing DDI microbump column (the sn35ag cap over the fraction
    1 - pillarH / standoff of the gap, on a Cu pillar) strained elastically (a 1e-9 s step) by
    1e-4 axially and in yz shear carries the series stresses 1e-4 / (f_s / E_s + f_p / E_p) and
    1e-4 / (f_s / G_s + f_p / G_p), with no in-plane stress: the published departures 1.6e-13 and
    5.5e-14 (rounding level; the oracle's Newton, restated in the reference's operation order,
    lands on the same digits)."""
    from tmsolve.materials import iso_modulus, iso_tables
    recs = json.load(open(GOLDEN))
    st = pm.default_stack()
    sn, cu = recs[st["ddi"]["solder"]], recs["cu"]
    pv = lambda o: o["v"] if isinstance(o, dict) else o
    nu_s, nu_p = pv(sn["elastic"]["nu"]), pv(cu["elastic"]["nu"])
    params = [pv(sn["anand"][k]) for k in ("A", "QR", "xi", "m", "shat", "n", "h0", "a", "s0")] + [nu_s]
    Etab = iso_tables(sn)["E"]
    fs = 1 - st["ddi"]["pillarH"] / st["ddi"]["standoff"]
    Es, Ep = iso_modulus(sn, 25.0), iso_modulus(cu, 25.0)
    Gs, Gp = Es / (2 * (1 + nu_s)), Ep / (2 * (1 + nu_p))
    state = np.zeros(12)
    state[6] = params[8]                               # s = s0
    eps = np.zeros(6)
    _, sig, _ = oracle_lib.anand_series_step(params, Etab, state, eps, [1e-4, 1e-4, 0.0], fs, [1 / Ep, 1 / Gp, 1 / Gp], 25.0, 1e-9)
    s_ref, t_ref = 1e-4 / (fs / Es + (1 - fs) / Ep), 1e-4 / (fs / Gs + (1 - fs) / Gp)
    ser = max(abs(sig[2] - s_ref) / s_ref, abs(sig[4] - t_ref) / t_ref)
    inplane = max(abs(sig[0]), abs(sig[1]), abs(sig[3])) / s_ref
    assert f"{ser:.1e}" == "1.6e-13" and f"{inplane:.1e}" == "5.5e-14", (ser, inplane)
