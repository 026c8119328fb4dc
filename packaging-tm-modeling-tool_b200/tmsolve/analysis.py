"""The process chain of the tool's analysis, on the host: the
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
from .pkgmesh import STAGE, build_package_mesh
from .thermal import band_section, group_step, group_tables, section_step, thermal_path_points

SOLIDUS_DEFAULT = 217.0


def _groups(cfg: dict, g: dict) -> list:
    """The homogeneous groups in packageGroups order (06-mesher.js:310-345), each dict(mat: record
    id, stage: birth stage, column: separate columns, si: silicon model, series: (record id, height
    fraction) of a second material in series along the columns): solder (stage 1, columns),
    underfill (2), the dies (1), then TIM, lid and lid adhesive or stiffener and its adhesive (3);
    with stacked modules, per module its chiplets, Si base and TSV Cu, then the DDI microbumps (a
    solder cap on a Cu pillar), all born at chiplet join (-3), the wafer underfill (-2) and the
    wafer mold (-1)."""
    grp = lambda mat, stage, column=False, si=None, series=None: dict(mat=mat, stage=stage, column=column, si=si, series=series)
    out = [grp(cfg["bump"]["solder"], 1, True), grp(cfg["underfill"]["mat"], 2)]
    for dc in cfg["dies"]:
        out.append(grp("si", 1, si=dc.get("si", "aniso")))
    if g["lid"]:
        L = cfg["lid"]
        out += [grp(L["timMat"], 3), grp(L["mat"], 3), grp(L["adhMat"], 3)]
    if g["stiff"]:
        S = cfg["stiffener"]
        out += [grp(S["mat"], 3), grp(S["adhMat"], 3)]
    if g["modules"]:
        st, S = cfg["stack"], STAGE
        for m in g["modules"]:
            out += [grp("si", S["DDI"], si=c["si"]) for c in m["chiplets"]]
            out.append(grp("si", S["DDI"], si=m["si"]))
            if m["tsv"] > 0:
                out.append(grp("cu", S["DDI"]))
        out.append(grp(st["ddi"]["solder"], S["DDI"], column=True, series=("cu", st["ddi"]["pillarH"] / st["ddi"]["standoff"])))
        if g["wcuf"]:
            out.append(grp(st["wcuf"]["mat"], S["WCUF"]))
        out.append(grp(st["moldMat"], S["MOLD"]))
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
    tabs = [group_tables(recs[h["mat"]], column=h["column"], si_model=h["si"] or "aniso",
                         series=(recs[h["series"][0]], h["series"][1]) if h["series"] else None) for h in hom]
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
                   group_stage=np.array([0] + [h["stage"] for h in hom], np.int32),
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
    for h in pkg.meta["groups"]:
        if stage is None or h["stage"] <= stage:
            add(h["mat"])
    if stage is None or stage >= 0:
        for r in cfg["substrate"]["layers"]:
            add(r.get("mat"))
            add(r.get("fill"))
    return out


def _module_segments(cfg: dict) -> tuple:
    """buildPath's stacked-module segments (11-analysis.js:169-175): chiplet join T_ddi -> T_fill
    (the wafer underfill's cure temperature, or the mold's for a mold-only fill) in stage DDI, then
    T_wcuf -> T_mold in stage WCUF (wafer underfill only) and T_mold -> T_sub in stage MOLD.
    Returns (the join segment, the segments after it)."""
    if not cfg.get("modules"):
        return [], []
    st, S = cfg["stack"], STAGE
    mp = st["process"]
    wcuf = st["fill"] == "wcuf"
    join = [(mp["Tddi"], mp["Twcuf"] if wcuf else mp["Tmold"], S["DDI"])]
    rest = ([(mp["Twcuf"], mp["Tmold"], S["WCUF"])] if wcuf else []) + [(mp["Tmold"], cfg["process"]["Tsub"], S["MOLD"])]
    return join, rest


def process_chain(pkg: Package, recs: dict) -> list:
    """The chain of buildPath (11-analysis.js:146-182): (Ta, Tb, stage) of every step from the
    first process temperature to 25 degC: the stacked modules' stages first (when the package
    has any), then the substrate's."""
    cfg = pkg.meta["cfg"]
    p = cfg["process"]
    stops = _solidi(pkg, recs)
    final = 2 if cfg["packageType"] == "bare" else 3
    join, mrest = _module_segments(cfg)
    segs = join + mrest
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


def _solidi(pkg: Package, recs: dict) -> list:
    """The path's solidus stops (11-analysis.js:127-130): the flip chip solder's, and the DDI
    microbump solder's when the package has stacked modules and its record gives one."""
    out = [_solidus(pkg, recs)]
    cfg = pkg.meta["cfg"]
    if cfg.get("modules"):
        sol = recs[cfg["stack"]["ddi"]["solder"]].get("solidus")
        if sol is not None:
            out.append(float(sol["v"] if isinstance(sol, dict) else sol))
    return out


def evaluation_temperatures(pkg: Package, recs: dict) -> dict:
    """evaluationTemperatures (11-analysis.js:132-144) of a full analysis: the cycling samples
    (with 25 degC) and the reflow sweep above the cycling range (every 15 degC, 10 degC near a
    glass transition, the solidus and one degree above it, the report temperatures, the peak)."""
    cfg = pkg.meta["cfg"]
    tgs = stage_tgs(pkg, recs)
    cyc = temperature_samples(cfg["cycling"]["Tmin"], cfg["cycling"]["Tmax"], tgs, [25])
    peak = cfg["reflow"]["peak"]
    ref = {25, peak, *cfg["reflow"]["reportTemps"]}
    for sol in _solidi(pkg, recs):
        ref |= {sol, sol + 1}
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
    """buildPath (11-analysis.js:146-182) of a full analysis, in its solve order: the stacked
    modules' chiplet join, its 'ddi' branch (T_fill -> 25 degC in stage DDI) and the module fill
    and mold cures (when the package has modules), the chain's S0 and S1 steps, the chip-join
    branch (T_UF -> 25 degC in S1), the rest of the chain, then the sweep branches in the final
    stage from 25 degC down to the coldest and up to the hottest evaluation temperature, stopping
    at every one. Returns dict(steps: [(Ta, Tb, stage, branch)], chain, cpi, down, up, ddiJoin,
    ddi: step indices, temps)."""
    cfg = pkg.meta["cfg"]
    p = cfg["process"]
    fin = 2 if cfg["packageType"] == "bare" else 3
    temps = evaluation_temperatures(pkg, recs)
    solidi = _solidi(pkg, recs)
    steps = []

    def seg(Ta, Tb, stage, branch, stops=()):
        pts = thermal_path_points(float(Ta), float(Tb), stage_tgs(pkg, recs, stage), list(stops) + solidi)
        ids = []
        for a, b in zip(pts[:-1], pts[1:]):
            steps.append((a, b, stage, branch))
            ids.append(len(steps) - 1)
        return ids
    # stacked modules first: chiplet join, the 'ddi' branch (the joined module cooled to 25 degC before
    # its fill is born), then the fill and mold cures up to the substrate's stress-free temperature
    join, mrest = _module_segments(cfg)
    sm_join = [k for (Ta, Tb, st) in join for k in seg(Ta, Tb, st, "chain")]
    ddi = seg(join[0][1], 25, STAGE["DDI"], "ddi") if join else []
    sm = sm_join + [k for (Ta, Tb, st) in mrest for k in seg(Ta, Tb, st, "chain")]
    s0 = seg(p["Tsub"], p["Tjoin"], 0, "chain") if abs(p["Tsub"] - p["Tjoin"]) > 1e-9 else []
    s1 = seg(p["Tjoin"], p["Tuf"], 1, "chain")
    cpi = seg(p["Tuf"], 25, 1, "cpi")
    rest = seg(p["Tuf"], p["Tattach"], 2, "chain") + seg(p["Tattach"], 25, 3, "chain") if fin == 3 else seg(p["Tuf"], 25, 2, "chain")
    ev = temps["all"]
    down = seg(25, min([25] + ev), fin, "down", ev)
    up = seg(25, max([25] + ev), fin, "up", ev)
    return dict(steps=steps, chain=sm + s0 + s1 + rest, cpi=cpi, down=down, up=up, temps=temps, ddiJoin=sm_join, ddi=ddi)


def solve_chain(model, pkg: Package, steps: list, tol: float = 1e-8, state_elems=None, state_f32: bool = True, **solve_kw):
    """Each step assembled and solved on a model (``assemble``/``assemble_step`` and ``solve``:
    the oracle's ``OracleModel`` or the library's ``DeviceModel``), as ``Analysis.run`` does
    (src/core/11-analysis.js:209-214, ``finishPath`` :230-256): the increments summed in double
    precision give the state at the chain's end (25 degC). With state_elems, the element history
    states of those elements are marched along (``accumulateStep``), rows of
    ``post.state_stride`` values, from the increments as the analysis keeps them for its element
    histories: rounded to float32 (``finishPath``), or in double precision with state_f32=False
    (the increments of ``solveStep`` used directly). Returns (u, solve records, states or None)."""
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
        u += r["u"]
        recs.append(r)
        if S is not None:
            du = r["u"].astype(np.float32).astype(np.float64) if state_f32 else r["u"]
            model.set_sublayers(step)
            model.accumulate_state(du, state_elems, stride, S)
    return u, recs, (S.reshape(-1, stride) if S is not None else None)
