"""The process chain of the tool's analysis for packages of monolithic dies, on the host: the
model that ``Analysis.build`` makes (src/core/11-analysis.js:100-113: ``buildPackageMesh``, then
``FEModel`` with the configuration's materials) and the chain of ``buildPath`` (:146-175), whose
summed increments are the as-assembled state at 25 degC:

* S0 T_sub -> T_join (the substrate alone, only when the two differ), S1 T_join -> T_UF (dies and
  solder joined), then S2 T_UF -> T_attach (underfill) and S3 T_attach -> 25 degC (lid or
  stiffener); a bare package cools T_UF -> 25 degC in S2;
* each segment in the steps of ``thermalPathPoints`` with the glass transitions of the materials
  born by its stage (``modelTgs``, :18-26) and the solder's solidus as a stop;
* every step: ``prepareStep`` data from the records' 1 degC tables (``thermal.py``), unborn groups
  at 1e-6 of their stiffness and without load (the solver's stage handling).

The materials are database records handed in by the caller (the tool's database stays on its
side); ``process_package`` builds the library's ``Package`` of that model, ``process_chain`` the
steps, and ``solve_chain`` runs them through a model object (the library's ``DeviceModel`` or the
oracle) and sums the increments.
"""
from __future__ import annotations

import math
from typing import Optional

import numpy as np

from .materials import material_tgs
from .packages import Package, StepData
from .pkgmesh import build_package_mesh
from .thermal import band_section, group_step, group_tables, section_step, thermal_path_points

SOLIDUS_DEFAULT = 217.0


def _groups(cfg: dict, g: dict) -> list:
    """(record id, birth stage, column phase, silicon model) of the homogeneous groups in packageGroups order
    (06-mesher.js:310-322): solder (stage 1, separate columns), underfill (2), the dies (1), then
    TIM, lid and lid adhesive or stiffener and its adhesive (3)."""
    out = [(cfg["bump"]["solder"], 1, True, None), (cfg["underfill"]["mat"], 2, False, None)]
    for d, dc in zip(g["dies"], cfg["dies"]):
        out.append(("si", 1, False, dc.get("si", "aniso")))
    if g["lid"]:
        L = cfg["lid"]
        out += [(L["timMat"], 3, False, None), (L["mat"], 3, False, None), (L["adhMat"], 3, False, None)]
    if g["stiff"]:
        S = cfg["stiffener"]
        out += [(S["mat"], 3, False, None), (S["adhMat"], 3, False, None)]
    return out


def process_package(cfg: dict, recs: dict, preset: str = "draft", override: Optional[dict] = None) -> Package:
    """The analysis model of a configuration at a mesh preset: the restated mesh, the substrate as
    one layered group over its bands (``buildBandSection`` of each band's rows), and one
    homogeneous group per part with its record's tables; groups born in their process stages."""
    mesh, info = build_package_mesh(cfg, dict(override or {}, preset=preset))
    g = info["geometry"]
    sub = g["sub"]
    bands = sub["bands"]
    secs = []
    for b in bands:
        subs = [(r["row"], max(b["z0"], r["z0"]), min(b["z1"], r["z1"])) for r in sub["rows"]
                if min(b["z1"], r["z1"]) - max(b["z0"], r["z0"]) > 1e-12]
        secs.append(band_section(b, subs, recs))
    nb = len(secs)
    sec_of_layer = np.zeros(mesh.nz - 1, np.int32)
    for k in range(mesh.nz - 1):
        zc = 0.5 * (mesh.zs[k] + mesh.zs[k + 1])
        for q, b in enumerate(bands):
            if b["z0"] < zc < b["z1"]:
                sec_of_layer[k] = q
    hom = _groups(cfg, g)
    tabs = [group_tables(recs[mid], column=col, si_model=si or "aniso") for (mid, _, col, si) in hom]
    n = nb + len(hom)

    def step_fn(Ta, Tb):
        W, V, D, s0 = np.zeros(108 * n), np.zeros(18 * n), np.zeros(36 * n), np.zeros(6 * n)
        for q, sec in enumerate(secs):
            W[108 * q:108 * q + 108], V[18 * q:18 * q + 18] = section_step(sec, Ta, Tb)
        for q, tab in enumerate(tabs):
            p = nb + q
            D[36 * p:36 * p + 36], s0[6 * p:6 * p + 6] = group_step(tab, Ta, Tb)
        lay = np.zeros(n, np.int32)
        lay[:nb] = 1
        return StepData(layered=lay, D=D, s0=s0, W=W, V=V, born=np.ones(n, np.int32), sub_n=np.zeros(n, np.int32),
                        sub_z=np.zeros(0), sub_D=np.zeros(0), sub_s0=np.zeros(0))

    return Package(name=f"process model, {info['preset']} mesh", mesh=mesh,
                   group_layered=np.array([1] + [0] * len(hom), np.int32),
                   group_stage=np.array([0] + [st for (_, st, _, _) in hom], np.int32),
                   group_pset=np.array([0] + [nb + q for q in range(len(hom))], np.int32), sec_of_layer=sec_of_layer,
                   npset=n, step_fn=step_fn, Ta=float(cfg["process"]["Tattach"]), Tb=25.0,
                   meta=dict(mesh_info=info, cfg=cfg, groups=hom, bottom_plane=0,
                             bga=dict(sx=cfg["substrate"]["sx"], sy=cfg["substrate"]["sy"], inset=cfg["bga"]["inset"],
                                      pitch=cfg["bga"]["pitch"])))


def stage_tgs(pkg: Package, recs: dict, stage: Optional[int] = None) -> list:
    """modelTgs (11-analysis.js:18-26): the glass transitions of the materials of the groups born
    by a stage (all groups for None), and of the substrate's rows (born in stage 0)."""
    cfg = pkg.meta["cfg"]
    out, seen = [], set()

    def add(mid):
        if mid and mid not in seen:
            seen.add(mid)
            out.extend(material_tgs(recs[mid]))
    for (mid, st, _, _) in pkg.meta["groups"]:
        if stage is None or st <= stage:
            add(mid)
    if stage is None or stage >= 0:
        for r in cfg["substrate"]["layers"]:
            add(r.get("mat"))
            add(r.get("fill"))
    return out


def process_chain(pkg: Package, recs: dict) -> list:
    """The chain of buildPath (11-analysis.js:146-175): (Ta, Tb, stage) of every step from the
    substrate's stress-free temperature to 25 degC."""
    cfg = pkg.meta["cfg"]
    p = cfg["process"]
    sol = recs[cfg["bump"]["solder"]].get("solidus")
    stops = [float(sol["v"] if isinstance(sol, dict) else sol) if sol is not None else SOLIDUS_DEFAULT]
    final = 2 if cfg["packageType"] == "bare" else 3
    segs = []
    if abs(p["Tsub"] - p["Tjoin"]) > 1e-9:
        segs.append((p["Tsub"], p["Tjoin"], 0))
    segs.append((p["Tjoin"], p["Tuf"], 1))
    if final == 3:
        segs += [(p["Tuf"], p["Tattach"], 2), (p["Tattach"], 25.0, 3)]
    else:
        segs.append((p["Tuf"], 25.0, 2))
    steps = []
    for (Ta, Tb, st) in segs:
        pts = thermal_path_points(float(Ta), float(Tb), stage_tgs(pkg, recs, st), stops)
        steps += [(a, b, st) for a, b in zip(pts[:-1], pts[1:])]
    return steps


CYCLE_DT_STEP, CYCLE_DT_FINE, CYCLE_TG_BAND = 10.0, 5.0, 15.0     # 00-constants.js:106-108
REFLOW_DT, REFLOW_DT_FINE = 15.0, 10.0


def _js_round(x: float) -> float:
    return math.floor(x + 0.5)


def temperature_samples(Tmin: float, Tmax: float, tgs, extras=()) -> list:
    """temperatureSamples (11-analysis.js:29-40): every 10 degC, every 5 degC within 15 degC of a
    glass transition, both ends and the extras, rounded to 1e-3 degC, ascending."""
    out = set()

    def add(T):
        if Tmin - 1e-9 <= T <= Tmax + 1e-9:
            out.add(_js_round(T * 1000) / 1000)
    add(Tmin)
    add(Tmax)
    T = math.ceil(Tmin / CYCLE_DT_STEP) * CYCLE_DT_STEP
    while T <= Tmax:
        add(T)
        T += CYCLE_DT_STEP
    for tg in tgs:
        T = math.ceil((tg - CYCLE_TG_BAND) / CYCLE_DT_FINE) * CYCLE_DT_FINE
        while T <= tg + CYCLE_TG_BAND:
            add(T)
            T += CYCLE_DT_FINE
    for T in extras:
        add(T)
    return sorted(out)


def _solidus(pkg: Package, recs: dict) -> float:
    sol = recs[pkg.meta["cfg"]["bump"]["solder"]].get("solidus")
    return float(sol["v"] if isinstance(sol, dict) else sol) if sol is not None else SOLIDUS_DEFAULT


def evaluation_temperatures(pkg: Package, recs: dict) -> dict:
    """evaluationTemperatures (11-analysis.js:132-144) of a full analysis: the cycling samples
    (with 25 degC) and the reflow sweep above the cycling range (every 15 degC, 10 degC near a
    glass transition, the solidus and one degree above it, the report temperatures, the peak)."""
    cfg = pkg.meta["cfg"]
    tgs = stage_tgs(pkg, recs)
    cyc = temperature_samples(cfg["cycling"]["Tmin"], cfg["cycling"]["Tmax"], tgs, [25])
    peak = cfg["reflow"]["peak"]
    sol = _solidus(pkg, recs)
    ref = {25, peak, sol, sol + 1, *cfg["reflow"]["reportTemps"]}
    T = math.ceil(cfg["cycling"]["Tmax"] / REFLOW_DT) * REFLOW_DT
    while T <= peak:
        ref.add(T)
        T += REFLOW_DT
    for tg in tgs:
        T = math.ceil((tg - CYCLE_TG_BAND) / REFLOW_DT_FINE) * REFLOW_DT_FINE
        while T <= tg + CYCLE_TG_BAND:
            ref.add(T)
            T += REFLOW_DT_FINE
    ref = sorted(float(T) for T in ref if 25 <= T <= peak)
    return dict(all=sorted(set(cyc) | set(ref)), cycling=cyc, reflow=ref)


def full_path(pkg: Package, recs: dict) -> dict:
    """buildPath (11-analysis.js:146-175) of a full analysis of monolithic dies, in its solve order:
    the chain's S0 and S1 steps, the chip-join branch (T_UF -> 25 degC in S1), the rest of the
    chain, then the sweep branches in the final stage from 25 degC down to the coldest and up to
    the hottest evaluation temperature, stopping at every one. Returns dict(steps: [(Ta, Tb,
    stage, branch)], chain, cpi, down, up: step indices, temps)."""
    cfg = pkg.meta["cfg"]
    p = cfg["process"]
    fin = 2 if cfg["packageType"] == "bare" else 3
    temps = evaluation_temperatures(pkg, recs)
    solidi = [_solidus(pkg, recs)]
    steps = []

    def seg(Ta, Tb, stage, branch, stops=()):
        pts = thermal_path_points(float(Ta), float(Tb), stage_tgs(pkg, recs, stage), list(stops) + solidi)
        ids = []
        for a, b in zip(pts[:-1], pts[1:]):
            steps.append((a, b, stage, branch))
            ids.append(len(steps) - 1)
        return ids
    s0 = seg(p["Tsub"], p["Tjoin"], 0, "chain") if abs(p["Tsub"] - p["Tjoin"]) > 1e-9 else []
    s1 = seg(p["Tjoin"], p["Tuf"], 1, "chain")
    cpi = seg(p["Tuf"], 25, 1, "cpi")
    rest = seg(p["Tuf"], p["Tattach"], 2, "chain") + seg(p["Tattach"], 25, 3, "chain") if fin == 3 else seg(p["Tuf"], 25, 2, "chain")
    ev = temps["all"]
    down = seg(25, min([25] + ev), fin, "down", ev)
    up = seg(25, max([25] + ev), fin, "up", ev)
    return dict(steps=steps, chain=s0 + s1 + rest, cpi=cpi, down=down, up=up, temps=temps)


def solve_chain(model, pkg: Package, steps: list, tol: float = 1e-8, state_elems=None, **solve_kw):
    """Each step assembled and solved on a model (``assemble``/``assemble_step`` and ``solve``:
    the oracle's ``OracleModel`` or the library's ``DeviceModel``). The increments are kept as
    float32, as the analysis stores them (src/core/11-analysis.js:256), and summed: the state at
    the chain's end (25 degC). With state_elems, the element history states of those elements are
    marched along (``accumulateStep``), rows of ``post.state_stride`` values. Returns (u, solve
    records, states or None)."""
    from .post import state_stride
    assemble = getattr(model, "assemble_step", None) or model.assemble
    u = np.zeros(3 * pkg.mesh.nn)
    recs, S, stride = [], None, 0
    if state_elems is not None:
        state_elems = np.ascontiguousarray(state_elems, np.int32)
        stride = state_stride(pkg.step(steps[0][0], steps[0][1], stage=steps[0][2]))
        S = np.zeros(stride * len(state_elems))
    for k, (a, b, st) in enumerate(steps):
        step = pkg.step(a, b, stage=st)
        r = model.solve(assemble(step), tol=tol, key=k, **solve_kw)
        du = r["u"].astype(np.float32).astype(np.float64)
        u += du
        recs.append(r)
        if S is not None:
            model.set_sublayers(step)
            model.accumulate_state(du, state_elems, stride, S)
    return u, recs, (S.reshape(-1, stride) if S is not None else None)
