"""Incremental thermoelastic steps of temperature-dependent materials, host side: the thermal
path the tool steps along and the per-step data of an isotropic material from its 1 degC tables.

* ``thermal_path_points`` restates ``thermalPathPoints`` (src/core/11-analysis.js:50-66): steps of
  at most 30 degC, 10 degC where a step would come within 15 degC of a glass transition, through
  the given stops;
* ``iso_step`` forms what ``FEModel.prepareStep`` (src/core/09-assembly.js:346-365) gives a
  homogeneous group of an isotropic table material: the stiffness averaged over the step
  (``gridMean``) and the thermal stress increment, the integral of D(T) dF(T) over the step
  (``gridStressIncrement``), with D(T) = E(T) D_1(nu);
* ``table_box_package``: a box of one such material (``boxModel``, src/core/15-verify.js:11-17)
  whose steps carry those data;
* substrate rows from database records on the 1 degC grid: a band's layered section
  (``buildBandSection``, src/core/04-homogenize.js:140-184: per sub-layer D_s(T) in plane-stress
  shell form and F_s(T), the weights W_j(T)) with its step data (``sectionWmean``, ``sectionVstep``,
  :206-221), and one row as a homogeneous orthotropic material (the 'rowmat' groups of
  ``FEModel._prepareGroup``, src/core/09-assembly.js:239-252).
"""
from __future__ import annotations

from typing import Optional

import numpy as np

from .materials import (NU_MAX_GLOBAL, TGRID_MIN, TGRID_N, T_STRAIN_ORIGIN, column_d, ec_d, for_grid_segments, grid_mean,
                        grid_modulus_strain_increment, iso_d, iso_modulus, iso_tables, lagrange3_integrals, material_ec,
                        material_tgs, silicon_d, sublayer_shell_d, substrate_row_ec, thermal_strain_at)
from .mesh import build_structured_mesh, constraints321
from .packages import CONSTRAINT_SPAN, Package, StepData, box_package

INC_DT_MAX = 30.0     # 00-constants.js:28
INC_DT_TG = 10.0
INC_TG_BAND = 15.0


def thermal_path_points(Ta: float, Tb: float, tgs, stops=()) -> list:
    """thermalPathPoints (11-analysis.js:50-66)."""
    d = float(np.sign(Tb - Ta))
    pts = [Ta]
    if d == 0:
        return pts
    inner = sorted((T for T in stops if (T - Ta) * d > 1e-9 and (Tb - T) * d > 1e-9), key=lambda T: d * T)
    inner.append(Tb)
    T = Ta
    for S in inner:
        while (S - T) * d > 1e-9:
            lo, hi = min(T, T + d * INC_DT_MAX), max(T, T + d * INC_DT_MAX)
            h = INC_DT_TG if any(tg + INC_TG_BAND > lo and tg - INC_TG_BAND < hi for tg in tgs) else INC_DT_MAX
            nxt = round((T + d * h) * 1e6) / 1e6
            T = nxt if (S - nxt) * d > 1e-9 else S
            pts.append(T)
    return pts


def iso_step(tab: dict, Ta: float, Tb: float):
    """(D 36, s0 6) of an isotropic table material over the step Ta -> Tb."""
    nu = min(tab["nu"], NU_MAX_GLOBAL)
    D1 = iso_d(1.0, nu)
    D = D1 * grid_mean(tab["E"], Ta, Tb)
    eF = grid_modulus_strain_increment(tab["E"], tab["F"], Ta, Tb)
    D1m = D1.reshape(6, 6)
    s0 = (D1m[:, 0] + D1m[:, 1] + D1m[:, 2]) * eF
    return D, s0


def table_box_package(mat: dict, xs, ys, zs, constraints=None, name="table box") -> Package:
    """A box of one isotropic table material (one homogeneous group), steps from its tables."""
    tab = iso_tables(mat)
    pkg = box_package(xs, ys, zs, [(iso_d(1.0, 0.3), 0.0, 0.0)], lambda i, j, k: 0, name=name, constraints=constraints)

    def step_fn(Ta, Tb):
        D, s0 = iso_step(tab, Ta, Tb)
        return StepData(layered=np.zeros(1, np.int32), D=D, s0=s0, W=np.zeros(108), V=np.zeros(18),
                        born=np.ones(1, np.int32), sub_n=np.zeros(1, np.int32), sub_z=np.zeros(0), sub_D=np.zeros(0),
                        sub_s0=np.zeros(0))
    pkg.step_fn = step_fn
    pkg.meta["tables"] = tab
    return pkg


# ---- substrate rows on the 1 degC grid -------------------------------------------------------

def _grid_vec(G: np.ndarray, T: float) -> np.ndarray:
    """gridAddAt's interpolation (03-materials.js:358-363) of a (TGRID_N, m) grid."""
    x = min(max(T - TGRID_MIN, 0.0), TGRID_N - 1)
    i = min(int(np.floor(x)), TGRID_N - 2)
    t = x - i
    return G[i] + t * (G[i + 1] - G[i])


def grid_mean_vec(G: np.ndarray, Ta: float, Tb: float) -> np.ndarray:
    """gridMean (03-materials.js:380-387) of a (TGRID_N, m) grid over the step [Ta, Tb]."""
    L = abs(Tb - Ta)
    if L < 1e-12:
        return _grid_vec(G, Ta).copy()
    out = np.zeros(G.shape[1])

    def seg(tm, t0, t1):
        out[:] += (t1 - t0) / L * _grid_vec(G, tm)
    for_grid_segments(Ta, Tb, seg)
    return out


def grid_stress_increment(Dg: np.ndarray, Fg: np.ndarray, Ta: float, Tb: float) -> np.ndarray:
    """gridStressIncrement (03-materials.js:394-411) for a stiffness grid (TGRID_N, 36) and a
    thermal strain grid (TGRID_N, 3): the integral from Ta to Tb of D(T) dF(T)."""
    sg = 1.0 if Tb >= Ta else -1.0
    out = np.zeros(6)

    def seg(tm, t0, t1):
        D = _grid_vec(Dg, tm).reshape(6, 6)
        f = _grid_vec(Fg, t1) - _grid_vec(Fg, t0)
        out[:] += sg * (D[:, 0] * f[0] + D[:, 1] * f[1] + D[:, 2] * f[2])
    for_grid_segments(Ta, Tb, seg)
    return out


def row_ec(row: dict, recs: dict, T: float) -> dict:
    """substrateRowEC (04-homogenize.js:35-54) at T from database records (recs: id -> record)."""
    ids = {"cu"} | {row[k] for k in ("mat", "fill") if k in row}
    return substrate_row_ec(row, {mid: material_ec(recs[mid], T) for mid in ids})


def row_tables(row: dict, recs: dict, nu_max: float = NU_MAX_GLOBAL, shell: bool = False):
    """A substrate row's stiffness D(T) (TGRID_N, 36; plane-stress shell form for a sub-layer of a
    layered band) and thermal strain F(T) (TGRID_N, 3; Simpson per 1 degC step on the homogenized
    CTE at T, T + 0.5, T + 1, shifted so that F(25) = 0)."""
    al = np.array([[e["ax"], e["ay"], e["az"]] for e in (row_ec(row, recs, TGRID_MIN + 0.5 * k) for k in range(2 * TGRID_N - 1))])
    F = np.zeros((TGRID_N, 3))
    for i in range(1, TGRID_N):
        F[i] = F[i - 1] + (al[2 * (i - 1)] + 4 * al[2 * i - 1] + al[2 * i]) / 6
    F -= F[int(T_STRAIN_ORIGIN - TGRID_MIN)].copy()
    D = np.zeros((TGRID_N, 36))
    for i in range(TGRID_N):
        d = ec_d(row_ec(row, recs, float(TGRID_MIN + i)), nu_max)
        D[i] = sublayer_shell_d(d) if shell else d
    return D, F


def band_section(band: dict, subs: list, recs: dict, nu_max: float = NU_MAX_GLOBAL) -> dict:
    """buildBandSection (04-homogenize.js:140-184): subs are the (row, z0, z1) pieces of the band;
    W(T) (TGRID_N, 108) = per j the sum over sub-layers of D_s(T) times the integral of the quadratic
    Lagrange basis L_j over the sub-layer."""
    h = band["z1"] - band["z0"]
    Ls = [lagrange3_integrals(2 * (z0 - band["z0"]) / h - 1, 2 * (z1 - band["z0"]) / h - 1) for (_, z0, z1) in subs]
    tabs = [row_tables(r, recs, nu_max, shell=True) for (r, _, _) in subs]
    W = np.zeros((TGRID_N, 108))
    for (D, _), L in zip(tabs, Ls):
        for j in range(3):
            W[:, 36 * j:36 * j + 36] += D * L[j]
    return dict(z0=band["z0"], z1=band["z1"], Ls=Ls, tabs=tabs, W=W)


def section_step(sec: dict, Ta: float, Tb: float):
    """(W 108, V 18) of a band section over the step: sectionWmean and sectionVstep
    (04-homogenize.js:206-221), V_j = sum_s (integral of D_s dF_s) times the integral of L_j."""
    W = grid_mean_vec(sec["W"], Ta, Tb)
    V = np.zeros(18)
    for (D, F), L in zip(sec["tabs"], sec["Ls"]):
        s0 = grid_stress_increment(D, F, Ta, Tb)
        for j in range(3):
            V[6 * j:6 * j + 6] += s0 * L[j]
    return W, V


def _step_data(n, layered, D=None, s0=None, W=None, V=None) -> StepData:
    z = np.zeros
    return StepData(layered=np.full(n, 1 if layered else 0, np.int32), D=z(36 * n) if D is None else D,
                    s0=z(6 * n) if s0 is None else s0, W=z(108 * n) if W is None else W, V=z(18 * n) if V is None else V,
                    born=np.ones(n, np.int32), sub_n=np.zeros(n, np.int32), sub_z=z(0), sub_D=z(0), sub_s0=z(0))


def substrate_box(xs, ys, rows_top_down: list, recs: dict, nb: int, per_row: bool = False, nu_max: float = NU_MAX_GLOBAL) -> Package:
    """A free substrate box of database-record rows (the two models of the reference's check V5,
    src/core/15-verify.js:205-235): the rows' substrate bands (``substrateBands`` with nb bands per
    group) as one layered group, one element layer per band (per_row False); or every physical
    row as its own homogeneous orthotropic group, one element layer per row (per_row True). 3-2-1
    constraints as ``boxModel``; steps carry the tables' step data."""
    from .pkgmesh import substrate_bands
    sb = substrate_bands(rows_top_down, nb)
    rows = sb["rows"]
    if per_row:
        zs = [0.0] + [r["z1"] for r in rows]
        tabs = [row_tables(r["row"], recs, nu_max) for r in rows]
        n = len(rows)

        def step_fn(Ta, Tb):
            D, s0 = np.zeros(36 * n), np.zeros(6 * n)
            for q, (Dg, Fg) in enumerate(tabs):
                D[36 * q:36 * q + 36] = grid_mean_vec(Dg, Ta, Tb)
                s0[6 * q:6 * q + 6] = grid_stress_increment(Dg, Fg, Ta, Tb)
            return _step_data(n, False, D=D, s0=s0)
        group_of_layer, layered, sec_of_layer = list(range(n)), np.zeros(n, np.int32), np.zeros(n, np.int32)
    else:
        zs = list(sb["planes"])
        secs = []
        for b in sb["bands"]:
            subs = [(r["row"], max(b["z0"], r["z0"]), min(b["z1"], r["z1"])) for r in rows
                    if min(b["z1"], r["z1"]) - max(b["z0"], r["z0"]) > 1e-12]
            secs.append(band_section(b, subs, recs, nu_max))
        n = len(secs)

        def step_fn(Ta, Tb):
            W, V = np.zeros(108 * n), np.zeros(18 * n)
            for q, sec in enumerate(secs):
                W[108 * q:108 * q + 108], V[18 * q:18 * q + 18] = section_step(sec, Ta, Tb)
            return _step_data(n, True, W=W, V=V)
        group_of_layer, layered, sec_of_layer = [0] * n, np.ones(1, np.int32), np.arange(n, dtype=np.int32)
    nx, ny, nz = len(xs), len(ys), len(zs)
    nc = (nx - 1) * (ny - 1) * (nz - 1)
    cg = np.full(2 * nc, -1, np.int32)
    cs = np.zeros(2 * nc)
    k = np.arange(nc) % (nz - 1)
    cg[0::2] = np.asarray(group_of_layer, np.int32)[k]
    cs[0::2] = 1.0
    mesh = build_structured_mesh(xs, ys, zs, cg, np.zeros(2 * nc, np.int32), cs)
    mesh.constraints = constraints321(mesh, CONSTRAINT_SPAN * min((xs[-1] - xs[0]) / 2, (ys[-1] - ys[0]) / 2))
    ng = len(layered)
    return Package(name="substrate box" + (" per row" if per_row else ""), mesh=mesh, group_layered=layered,
                   group_stage=np.zeros(ng, np.int32), group_pset=np.arange(ng, dtype=np.int32), sec_of_layer=sec_of_layer,
                   npset=n, step_fn=step_fn, Ta=25.0, Tb=125.0)


# ---- homogeneous groups of database records ----------------------------------------------------

def group_tables(mat: dict, column: bool = False, si_model: str = "aniso", nu_max: float = NU_MAX_GLOBAL,
                 series: Optional[tuple] = None) -> dict:
    """FEModel._prepareGroup (09-assembly.js:253-284) for a homogeneous group of one record: the
    thermal strains F(T) (TGRID_N, 3: in-plane twice, through-thickness) and either a constant
    stiffness (cubic silicon, an isotropic record of constant modulus without a solidus) or a
    stiffness grid (TGRID_N, 36): isotropic D(E(T), nu) (the solder phase as separate columns,
    ``column``), orthotropic from the record's constants at T. ``series`` = (record, f): the
    columns are a cap of this record on a pillar of the other over the height fraction f
    (``_seriesColumn``, :288-305): compliances add by height, 1/E = (1 - f)/E_s + f/E_p and
    1/G likewise, columnD(E, E / 2G - 1), F = (1 - f) F_s + f F_p."""
    cxy = mat.get("cteXY") or mat["cte"]
    cz = mat.get("cteZ") or cxy
    F = np.zeros((TGRID_N, 3))
    for i in range(TGRID_N):
        T = float(TGRID_MIN + i)
        fxy = thermal_strain_at(cxy, T)
        F[i] = (fxy, fxy, fxy if cz is cxy else thermal_strain_at(cz, T))
    el = mat["elastic"]
    if el["type"] == "cubic":
        return dict(Dconst=silicon_d(si_model), F=F)
    if el["type"] == "iso":
        nu = el["nu"]["v"] if isinstance(el["nu"], dict) else el["nu"]
        mk = (lambda E: column_d(E, nu)) if column else (lambda E: iso_d(E, nu, nu_max))
        if series is not None:
            tp, fp = iso_tables(series[0]), series[1]
            Dg = np.zeros((TGRID_N, 36))
            for i in range(TGRID_N):
                Es, Ep = iso_modulus(mat, float(TGRID_MIN + i)), tp["E"][i]
                Gs, Gp = Es / (2 * (1 + nu)), Ep / (2 * (1 + tp["nu"]))
                E = 1 / ((1 - fp) / Es + fp / Ep)
                G = 1 / ((1 - fp) / Gs + fp / Gp)
                Dg[i] = column_d(E, E / (2 * G) - 1)
                F[i] = (1 - fp) * F[i] + fp * tp["F"][i]
            return dict(Dgrid=Dg, F=F)
        if el["E"]["type"] == "const" and mat.get("solidus") is None:
            return dict(Dconst=mk(iso_modulus(mat, float(TGRID_MIN))), F=F)
        return dict(Dgrid=np.array([mk(iso_modulus(mat, float(TGRID_MIN + i))) for i in range(TGRID_N)]), F=F)
    if el["type"] == "ortho":
        return dict(Dgrid=np.array([ec_d(material_ec(mat, float(TGRID_MIN + i)), nu_max) for i in range(TGRID_N)]), F=F)
    raise ValueError(f"elastic type {el['type']!r} not restated")


def group_step(tab: dict, Ta: float, Tb: float):
    """prepareStep (09-assembly.js:346-365) for a homogeneous group: (D 36, s0 6) of the step."""
    if "Dconst" in tab:
        Dc = tab["Dconst"].reshape(6, 6)
        f = _grid_vec(tab["F"], Tb) - _grid_vec(tab["F"], Ta)
        return tab["Dconst"].copy(), Dc[:, 0] * f[0] + Dc[:, 1] * f[1] + Dc[:, 2] * f[2]
    return grid_mean_vec(tab["Dgrid"], Ta, Tb), grid_stress_increment(tab["Dgrid"], tab["F"], Ta, Tb)
