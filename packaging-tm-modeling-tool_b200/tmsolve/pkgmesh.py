"""The tool's package mesher: the host-side restatement of
``buildPackageMesh`` (src/core/06-mesher.js:468-563) and what it needs, so that the reference's
own packages (its default lidded single die, its lid and stiffener variants) can be built and
solved through the library.

Restated from the reference, in the reference's arithmetic order where a floating-point result
decides a grid line or an element:

* the configuration's geometry fields: ``generateStack`` (src/core/02-config.js:24-56),
  ``defaultDie`` (:58-63) and ``defaultConfig`` (:140-166), geometry only (materials,
  process and post-processing settings are the caller's);
* ``substrateBands`` (src/core/04-homogenize.js:64-105): the build-up and core groups of the
  substrate, each split into ``layers`` bands of equal thickness;
* ``deriveGeometry`` (src/core/05-geometry.js:98-175): z levels, bump fields
  (``bumpAxis``, ``bumpFieldRects``, :23-58), underfill fillet, lid and stiffener footprints;
  ``wedgeHeight`` (:216-240), ``dieAt`` (:255-258), ``cellBumpFraction`` (:205-211);
* the mesher's in-plane grid (``axisFeatures`` :196-248, ``mergeFeatures`` :121-134,
  ``gridLines`` :142-189), z planes (``zPlanes`` :253-305), groups (``packageGroups`` :310-322),
  cell assignment (``makePackageAssign`` :344-453) and the DOF-cap loop of
  ``buildPackageMesh`` with its final refinement at the lid foot or stiffener ring edges.

Stacked modules with a Si base (``defaultModule``, ``defaultChiplet``, ``defaultStack``,
02-config.js:82-117; their geometry, feature lines, planes, groups, cells and three-point supports,
06-mesher.js:87-109, :209-222, :246-251, :281-286, :328-343, :376-427, :477-482, :534-545) are
restated too; organic RDL interposer bases are not (``stacked_module`` in ``packages.py`` is the
library's own module workload).
"""
from __future__ import annotations

import math
from typing import Optional

import numpy as np

from .mesh import PART, Mesh, build_structured_mesh, constraints321, module_support

# the mesher's constants (src/core/00-constants.js:34-55)
FEATURE_SNAP_TOL = 0.010
PLANE_MERGE_TOL = 0.001
GROWTH_RATIO_MAX = 1.3
REFINE_ZONE_FACTOR = 2.0
MIN_ELEMS_ACROSS_RING = 3
RING_EDGE_ZONE = 0
SLIVER_FRACTION = 0.125
MIN_ELEMS_ACROSS_FILLET = 6
FILLET_COL_MIN_FRACTION = 0.5
FILLET_FILL_SAMPLES = 4
FILLET_FILL_MIN = 0.05
SIZE_SAMPLES = 256
CAP_GROWTH_PAD = 1.03
CAP_MAX_ITER = 12
CONSTRAINT_SPAN = 0.4
MODULE_HMIN_PER_HEIGHT = 4
STAGE = dict(DDI=-3, WCUF=-2, MOLD=-1)      # the module process stages before the substrate's (00-constants.js:27)
MESH_PRESETS = {
    "draft": dict(label="Draft", hmin=0.6, hmax=3.0, cap=75000, layers=1),
    "standard": dict(label="Standard", hmin=0.25, hmax=1.5, cap=330000, layers=2),
    "fine": dict(label="Fine", hmin=0.10, hmax=0.6, cap=850000, layers=4),
}


def _clamp(x, lo, hi):
    """clamp (src/core/01-util.js:3)."""
    return lo if x < lo else (hi if x > hi else x)


def _simpson(f, a, b, n):
    """simpson (src/core/01-util.js:197-203)."""
    if n % 2:
        n += 1
    h = (b - a) / n
    s = f(a) + f(b)
    for i in range(1, n):
        s += f(a + i * h) * (4 if i % 2 else 2)
    return s * h / 3


# ---- configuration (geometry fields) -------------------------------------------------------

def generate_stack(**o) -> list:
    """generateStack (02-config.js:24-56): an N-2-N substrate, rows listed top to bottom (type,
    thickness; Cu rows with their residual ratio r, plane or signal kind and fill dielectric;
    dielectric, core and solder-resist rows with their material, the core with its plated
    through-hole Cu fraction). Per side, from the outer pad layer inwards: the pad layer
    (residual ratio rTopPad or rBottomPad), then plane and signal layers alternating."""
    p = dict(n=6, dielT=0.025, cuT=0.015, coreT=0.8, coreCuT=0.018, srT=0.020, pth=0.02, rPlane=0.75, rSignal=0.45,
             rTopPad=0.35, rBottomPad=0.55, rCoreCu=0.70, diel="abf_gl", core="mcl_e_795g", sr="psr4000")
    p.update(o)

    def side(pad_r):
        rows = []
        for k in range(p["n"]):
            kind = "signal" if k == 0 else ("plane" if k % 2 == 1 else "signal")
            r = pad_r if k == 0 else (p["rPlane"] if kind == "plane" else p["rSignal"])
            rows.append(dict(type="cu", t=p["cuT"], r=r, kind=kind, fill=p["diel"]))
            rows.append(dict(type="diel", t=p["dielT"], mat=p["diel"], via=0))
        return rows   # outer to inner

    rows = [dict(type="sr", t=p["srT"], mat=p["sr"])]
    rows += side(p["rTopPad"])
    if p["coreT"] > 0:
        rows += [dict(type="cu", t=p["coreCuT"], r=p["rCoreCu"], kind="plane", fill=p["diel"]),
                 dict(type="core", t=p["coreT"], mat=p["core"], pth=p["pth"]),
                 dict(type="cu", t=p["coreCuT"], r=p["rCoreCu"], kind="plane", fill=p["diel"])]
    rows += side(p["rBottomPad"])[::-1]
    rows.append(dict(type="sr", t=p["srT"], mat=p["sr"]))
    return rows


def default_die(did: str, x: float, y: float) -> dict:
    """defaultDie (02-config.js:58-63), geometry fields."""
    return dict(id=did, name="Die " + did.lstrip("D"), x=x, y=y, sx=20.0, sy=20.0, t=0.775, rot=0, si="aniso",
                bump=dict(type="full", rows=3, px=0.150, py=0.150, keepout=0.150, ubm=0.085, sro=0.090, dmax=0.105))


def default_chiplet(cid: str, x: float, y: float, sx: float = 10.0, sy: float = 10.0) -> dict:
    """defaultChiplet (02-config.js:82-84): a chiplet placed relative to its module."""
    return dict(id=cid, name="Chiplet " + cid.lstrip("C"), x=x, y=y, sx=sx, sy=sy, rot=0, si="aniso",
                ddi=dict(type="full", rows=3, keepout=0.050))


def default_module(mid: str, x: float, y: float) -> dict:
    """defaultModule (02-config.js:92-100) with a Si base: a 22 x 16 mm base 0.100 mm thick with
    1 % TSV Cu, on the flip chip bumps, carrying two 10 x 14 mm chiplets."""
    return dict(id=mid, name="Module " + mid.lstrip("M"), x=x, y=y, sx=22.0, sy=16.0, rot=0, base="si", tBase=0.100,
                si="aniso", tsv=0.01,
                bump=dict(type="full", rows=3, px=0.150, py=0.150, keepout=0.150, ubm=0.085, sro=0.090, dmax=0.105),
                chiplets=[default_chiplet("C1", -5.4, 0, 10.0, 14.0), default_chiplet("C2", 5.4, 0, 10.0, 14.0)])


def default_stack() -> dict:
    """defaultStack (02-config.js:108-117): the package-wide module technology (chiplet thickness,
    the DDI microbump: a Cu pillar under a solder cap, the DDI fill, the module process
    temperatures)."""
    return dict(chipletT=0.700, ddi=dict(standoff=0.025, pillarH=0.012, d=0.025, px=0.040, py=0.040, solder="sn35ag"),
                fill="wcuf", wcuf=dict(mat="cv5300", Wf=0.30, Hf=0.5), moldMat="ei6042",
                process=dict(Tddi=221, Twcuf=150, Tmold=180))


def default_config() -> dict:
    """defaultConfig (02-config.js:140-166): the lidded single-die package, its geometry, the
    material ids of its parts, the process temperatures and the BGA grid (materials database,
    reflow, cycling and post-processing settings are the caller's)."""
    return dict(
        substrate=dict(sx=45.0, sy=45.0, layers=generate_stack()),
        bga=dict(pitch=1.0, ballH=0.50, inset=1.0),
        packageType="lid",
        bump=dict(standoff=0.075, solder="sac305"),
        dies=[default_die("D1", 0.0, 0.0)],
        modules=[],
        stack=default_stack(),
        underfill=dict(mat="uf9000ae", Wf=0.8, Hf=0.7),
        lid=dict(mat="cu", ox=43.0, oy=43.0, tPlate=1.0, footW=3.0, adhMat="eccobond3005", adhT=0.100, timMat="tim_gel", blt=0.050),
        stiffener=dict(mat="cu", ox=53.0, oy=53.0, ringW=4.0, t=0.8, adhMat="eccobond3005", adhT=0.050),
        process=dict(Tsub=217, Tjoin=217, Tuf=165, Tattach=150),
        reflow=dict(peak=260, reportTemps=[25, 150, 220, 260]),
        cycling=dict(cond="G", Tmin=-40, Tmax=125),
        mesh=dict(preset="standard"),
    )


def preset_config(which: str, variant: Optional[str] = None) -> dict:
    """presetConfig (02-config.js:169-243), geometry fields: 'default', 'bare', 'stiffener2' (two
    dies side by side, stiffener ring), 'offset' (an offset bare die), 'coreStudy' (variant 'A':
    0.4 mm core, 'B': 0.8 mm core) and 'foveros' (a Si base die with three chiplets, lidded)."""
    c = default_config()
    if which == "default":
        pass
    elif which == "bare":
        c["packageType"] = "bare"
    elif which == "stiffener2":
        c["packageType"] = "stiffener"
        c["substrate"]["sx"] = c["substrate"]["sy"] = 55
        gap, w = 0.20, 16.0
        d1, d2 = default_die("D1", -(w + gap) / 2, 0), default_die("D2", (w + gap) / 2, 0)
        for d in (d1, d2):
            d["sx"], d["sy"] = 16.0, 24.0
        c["dies"] = [d1, d2]
        c["stiffener"] = dict(mat="cu", ox=53.0, oy=53.0, ringW=4.0, t=0.8, adhMat="eccobond3005", adhT=0.050)
    elif which == "offset":
        c["packageType"] = "bare"
        c["dies"][0].update(sx=15, sy=15, x=8, y=6)
    elif which == "coreStudy":
        v = "A" if variant == "A" else "B"
        c["packageType"] = "bare"
        c["substrate"]["sx"] = c["substrate"]["sy"] = 40
        c["substrate"]["layers"] = generate_stack(n=3, dielT=0.020, cuT=0.015, srT=0.019, coreT=0.4 if v == "A" else 0.8, coreCuT=0.015)
    elif which == "foveros":
        # one Si base die 0.150 mm thick with three chiplets, lidded
        m = default_module("M1", 0, 0)
        m.update(name="Base die 1", sx=21.0, sy=16.0, tBase=0.150, tsv=0.01)
        m["chiplets"] = [default_chiplet("C1", -5.15, 3.85, 10.0, 7.2), default_chiplet("C2", 5.15, 3.85, 10.0, 7.2),
                         default_chiplet("C3", 0, -3.85, 20.3, 7.2)]
        c["dies"] = []
        c["modules"] = [m]
        c["stack"]["chipletT"] = 0.700
    else:
        raise ValueError(f"preset {which!r} is not restated (the RDL-interposer presets are not)")
    return c


# ---- geometry ------------------------------------------------------------------------------

def substrate_bands(rows_top_down: list, nb: int) -> dict:
    """substrateBands (04-homogenize.js:64-105): z planes of the substrate's element bands."""
    rows = []
    z = 0.0
    for i in range(len(rows_top_down) - 1, -1, -1):
        r = rows_top_down[i]
        rows.append(dict(idx=i, row=r, z0=z, z1=z + r["t"]))
        z += r["t"]
    total = z
    core_at = next((q for q, r in enumerate(rows) if r["row"]["type"] == "core"), -1)
    if core_at >= 0:
        core = rows[core_at]
        below = rows[core_at - 1] if core_at > 0 and rows[core_at - 1]["row"]["type"] == "cu" else None
        above = rows[core_at + 1] if core_at + 1 < len(rows) and rows[core_at + 1]["row"]["type"] == "cu" else None
        z_lo = below["z0"] if below else core["z0"]
        z_hi = above["z1"] if above else core["z1"]
        groups = [(0.0, z_lo), (z_lo, z_hi), (z_hi, total)]
    else:
        groups = [(0.0, total)]
    cuts = [0.0]
    for z0, z1 in groups:
        for q in range(1, nb + 1):
            cuts.append(z0 + (z1 - z0) * q / nb)
    planes = [cuts[0]]
    for c in cuts[1:]:
        if c - planes[-1] > 1e-9:
            planes.append(c)
    bands = [dict(z0=planes[b], z1=planes[b + 1]) for b in range(len(planes) - 1)]
    return dict(total=total, rows=rows, planes=planes, bands=bands)


def bump_axis(c: float, L: float, k: float, p: float) -> dict:
    """bumpAxis (05-geometry.js:23-29)."""
    span0 = L - 2 * k
    if span0 < -1e-12 or p <= 0:
        return dict(n=0, first=c, last=c)
    n = math.floor(span0 / p + 1e-9) + 1
    span = (n - 1) * p
    return dict(n=n, first=c - span / 2, last=c + span / 2)


def bump_profile_deff(ubm: float, sro: float, dmax: float, H: float) -> float:
    """Effective diameter of a bump of truncated-sphere profile (bumpProfile,
    src/core/04-homogenize.js:282-307): the diameter of the cylinder of the same volume and height."""
    rt, rb = ubm / 2, sro / 2
    rm = max(dmax / 2, rt, rb)
    db, dt = rm - rb, rm - rt
    if db < 1e-12 and dt < 1e-12:
        zm, rho = H / 2, math.inf
    elif db < 1e-12:
        zm, rho = 0.0, (H * H + dt * dt) / (2 * dt)
    elif dt < 1e-12:
        zm, rho = H, (H * H + db * db) / (2 * db)
    else:
        g = lambda r: math.sqrt(max(0.0, 2 * r * db - db * db)) + math.sqrt(max(0.0, 2 * r * dt - dt * dt)) - H
        lo = max(db, dt) / 2
        hi = lo
        while g(hi) < 0:
            hi *= 2
        for _ in range(200):
            mid = 0.5 * (lo + hi)
            if g(mid) < 0:
                lo = mid
            else:
                hi = mid
        rho = 0.5 * (lo + hi)
        zm = math.sqrt(max(0.0, 2 * rho * db - db * db))

    def radius_at(z):
        if not math.isfinite(rho):
            return rm
        dz = z - zm
        return rm - rho + math.sqrt(max(0.0, rho * rho - dz * dz))

    volume = _simpson(lambda z: math.pi * radius_at(z) * radius_at(z), 0.0, H, 400)
    return math.sqrt(4 * volume / (math.pi * H))


def bump_field_rects(cx, cy, w, h, rect, bump, px, py) -> dict:
    """bumpFieldRects (05-geometry.js:45-58)."""
    ax, ay = bump_axis(cx, w, bump["keepout"], px), bump_axis(cy, h, bump["keepout"], py)
    field = None
    if ax["n"] > 0 and ay["n"] > 0:
        field = dict(x0=max(rect["x0"], ax["first"] - px / 2), x1=min(rect["x1"], ax["last"] + px / 2),
                     y0=max(rect["y0"], ay["first"] - py / 2), y1=min(rect["y1"], ay["last"] + py / 2))
    inner = None
    N = max(1, round(bump.get("rows", 1) or 1))
    if field and bump["type"] == "peripheral" and ax["n"] > 2 * N and ay["n"] > 2 * N:
        inner = dict(x0=ax["first"] + (N - 0.5) * px, x1=ax["last"] - (N - 0.5) * px,
                     y0=ay["first"] + (N - 0.5) * py, y1=ay["last"] - (N - 0.5) * py)
    return dict(nbx=ax["n"], nby=ay["n"], bx0=ax["first"], by0=ay["first"], field=field, inner=inner, rows=N,
                peripheral=inner is not None)


def derive_geometry(cfg: dict, layers: int) -> dict:
    """deriveGeometry (05-geometry.js:98-175): the monolithic dies, then the stacked modules (Si
    base only) with their chiplets; ``dies`` holds both (the objects on the flip chip bump layer),
    ``monoDies`` and ``modules`` each kind."""
    for m in cfg.get("modules") or []:
        if m.get("base", "si") == "rdl":
            raise ValueError("modules on an organic RDL interposer are not part of this mesher restatement")
    sub = substrate_bands(cfg["substrate"]["layers"], layers)
    zt = sub["total"]
    so = cfg["bump"]["standoff"]
    zaf = zt + so
    sx, sy = cfg["substrate"]["sx"], cfg["substrate"]["sy"]
    substrate = dict(x0=-sx / 2, x1=sx / 2, y0=-sy / 2, y1=sy / 2)
    dies = []
    for i, d in enumerate(cfg["dies"]):
        rot = d.get("rot", 0) == 90
        w, h = (d["sy"], d["sx"]) if rot else (d["sx"], d["sy"])
        b = d["bump"]
        px, py = (b["py"], b["px"]) if rot else (b["px"], b["py"])
        rect = dict(x0=d["x"] - w / 2, x1=d["x"] + w / 2, y0=d["y"] - h / 2, y1=d["y"] + h / 2)
        o = bump_field_rects(d["x"], d["y"], w, h, rect, b, px, py)
        deff = bump_profile_deff(b["ubm"], b["sro"], b["dmax"], so)
        abump = math.pi * deff * deff / 4
        o.update(index=i, kind="die", name=d["name"], rect=rect, cx=d["x"], cy=d["y"], w=w, h=h, px=px, py=py,
                 t=d["t"], zaf=zaf, ztop=zaf + d["t"], deff=deff, density=abump / (px * py))
        dies.append(o)
    mods = cfg.get("modules") or []
    st = cfg["stack"] if mods else None
    modules = []
    for mi, m in enumerate(mods):
        rot = m.get("rot", 0) == 90
        w, h = (m["sy"], m["sx"]) if rot else (m["sx"], m["sy"])
        b = m["bump"]
        px, py = (b["py"], b["px"]) if rot else (b["px"], b["py"])
        rect = dict(x0=m["x"] - w / 2, x1=m["x"] + w / 2, y0=m["y"] - h / 2, y1=m["y"] + h / 2)
        o = bump_field_rects(m["x"], m["y"], w, h, rect, b, px, py)
        deff = bump_profile_deff(b["ubm"], b["sro"], b["dmax"], so)
        abump = math.pi * deff * deff / 4
        t_base = m["tBase"]
        z_base_top = zaf + t_base
        z_ddi_top = z_base_top + st["ddi"]["standoff"]
        H = t_base + st["ddi"]["standoff"] + st["chipletT"]
        o.update(index=len(cfg["dies"]) + mi, kind="module", modIndex=mi, name=m["name"], rect=rect, cx=m["x"], cy=m["y"], w=w,
                 h=h, px=px, py=py, t=H, zaf=zaf, ztop=zaf + H, deff=deff, density=abump / (px * py), base="si",
                 tBase=t_base, zBaseTop=z_base_top, zDdiTop=z_ddi_top, si=m.get("si") or "aniso", tsv=max(0.0, m.get("tsv") or 0.0))
        # chiplets: centres rotated with the module, sizes and DDI pitch swapped by the module and the chiplet rotation
        dpx, dpy = st["ddi"]["px"], st["ddi"]["py"]
        a_ddi = math.pi * st["ddi"]["d"] * st["ddi"]["d"] / 4
        chips = []
        for ci, c in enumerate(m["chiplets"]):
            ccx, ccy = m["x"] + (-c["y"] if rot else c["x"]), m["y"] + (c["x"] if rot else c["y"])
            swap = rot != (c.get("rot", 0) == 90)
            cw, ch = (c["sy"], c["sx"]) if swap else (c["sx"], c["sy"])
            cpx, cpy = (dpy, dpx) if swap else (dpx, dpy)
            crect = dict(x0=ccx - cw / 2, x1=ccx + cw / 2, y0=ccy - ch / 2, y1=ccy + ch / 2)
            f = bump_field_rects(ccx, ccy, cw, ch, crect, c["ddi"], cpx, cpy)
            f.update(index=ci, modIndex=mi, name=m["name"] + " / " + c["name"], cx=ccx, cy=ccy, w=cw, h=ch, rect=crect, px=cpx,
                     py=cpy, t=st["chipletT"], si=c.get("si") or "aniso", zaf=z_ddi_top, zb=z_ddi_top,
                     ztop=z_ddi_top + st["chipletT"], deff=st["ddi"]["d"], abump=a_ddi, density=a_ddi / (cpx * cpy), kind="chiplet")
            chips.append(f)
        o["chiplets"] = chips
        modules.append(o)
    objs = dies + modules
    tmax = max((d["t"] for d in objs), default=0.0)
    g = dict(cfg=cfg, layers=layers, sub=sub, zt=zt, zaf=zaf, so=so, substrate=substrate, dies=objs, monoDies=dies,
             modules=modules, tmax=tmax, stack=st, uf=dict(Wf=cfg["underfill"]["Wf"], Hf=cfg["underfill"]["Hf"]), lid=None,
             stiff=None, wcuf=None)
    if st and st["fill"] == "wcuf":
        g["wcuf"] = dict(Wf=st["wcuf"]["Wf"], Hf=st["wcuf"]["Hf"])
    if cfg["packageType"] == "lid":
        L = cfg["lid"]
        outer = dict(x0=-L["ox"] / 2, x1=L["ox"] / 2, y0=-L["oy"] / 2, y1=L["oy"] / 2)
        inner = dict(x0=outer["x0"] + L["footW"], x1=outer["x1"] - L["footW"], y0=outer["y0"] + L["footW"],
                     y1=outer["y1"] - L["footW"])
        z_lid_bot = zaf + tmax + L["blt"]
        g["lid"] = dict(outer=outer, inner=inner, zAdhTop=zt + L["adhT"], zLidBot=z_lid_bot, zLidTop=z_lid_bot + L["tPlate"],
                        footH=so + tmax + L["blt"] - L["adhT"])
    if cfg["packageType"] == "stiffener":
        S = cfg["stiffener"]
        outer = dict(x0=-S["ox"] / 2, x1=S["ox"] / 2, y0=-S["oy"] / 2, y1=S["oy"] / 2)
        inner = dict(x0=outer["x0"] + S["ringW"], x1=outer["x1"] - S["ringW"], y0=outer["y0"] + S["ringW"],
                     y1=outer["y1"] - S["ringW"])
        g["stiff"] = dict(outer=outer, inner=inner, zAdhTop=zt + S["adhT"], zTop=zt + S["adhT"] + S["t"])
    return g


def _dist_to_rect(r, x, y):
    dx = max(r["x0"] - x, 0.0, x - r["x1"])
    dy = max(r["y0"] - y, 0.0, y - r["y1"])
    return math.hypot(dx, dy)


def wedge_height(objs, Wf, Hf, x, y):
    """wedgeHeight (05-geometry.js:216-240): fillet height at (x, y) and whether (x, y) is in a footprint."""
    h, in_fp = 0.0, False
    for d in objs:
        dist = _dist_to_rect(d["rect"], x, y)
        if dist <= Wf + 1e-12:
            in_fp = True
            if Wf > 0:
                h = max(h, Hf * d["t"] * (1 - dist / Wf))
    for a in range(len(objs)):
        for b in range(a + 1, len(objs)):
            A, B = objs[a]["rect"], objs[b]["rect"]
            tmin = min(objs[a]["t"], objs[b]["t"])
            oy0, oy1 = max(A["y0"], B["y0"]), min(A["y1"], B["y1"])
            ox0, ox1 = max(A["x0"], B["x0"]), min(A["x1"], B["x1"])
            gx = max(A["x0"] - B["x1"], B["x0"] - A["x1"])
            gy = max(A["y0"] - B["y1"], B["y0"] - A["y1"])
            if 0 < gx < Wf and oy1 > oy0 and oy0 <= y <= oy1:
                lo, hi = min(A["x1"], B["x1"]), max(A["x0"], B["x0"])
                if lo <= x <= hi:
                    in_fp = True
                    h = max(h, Hf * tmin)
            if 0 < gy < Wf and ox1 > ox0 and ox0 <= x <= ox1:
                lo, hi = min(A["y1"], B["y1"]), max(A["y0"], B["y0"])
                if lo <= y <= hi:
                    in_fp = True
                    h = max(h, Hf * tmin)
    return h, in_fp


def die_at(g, x, y):
    """dieAt (05-geometry.js:255-258): the die whose footprint strictly holds (x, y), or None."""
    for d in g["dies"]:
        r = d["rect"]
        if r["x0"] < x < r["x1"] and r["y0"] < y < r["y1"]:
            return d
    return None


def _point_in_rect(r, x, y):
    return r["x0"] <= x <= r["x1"] and r["y0"] <= y <= r["y1"]


def _rect_area(r):
    return max(0.0, r["x1"] - r["x0"]) * max(0.0, r["y1"] - r["y0"])


def _rect_intersect_area(a, b):
    w = min(a["x1"], b["x1"]) - max(a["x0"], b["x0"])
    h = min(a["y1"], b["y1"]) - max(a["y0"], b["y0"])
    return w * h if w > 0 and h > 0 else 0.0


def cell_bump_fraction(d, cell) -> float:
    """cellBumpFraction (05-geometry.js:205-211): bump area fraction of a cell under die d."""
    if not d["field"]:
        return 0.0
    a = _rect_intersect_area(cell, d["field"])
    if d["inner"]:
        a -= _rect_intersect_area(cell, d["inner"])
    ac = _rect_area(cell)
    return _clamp(a * d["density"] / ac, 0.0, 1.0) if ac > 0 else 0.0


# ---- in-plane grid -------------------------------------------------------------------------

def merge_features(feats: list, tol: float) -> dict:
    """mergeFeatures (06-mesher.js:121-134): feature lines closer than tol merged, the higher
    priority keeping its position (a stable sort by position first)."""
    feats = sorted(feats, key=lambda f: f["v"])
    out = []
    for f in feats:
        last = out[-1] if out else None
        if last is not None and f["v"] - last["v"] < tol:
            if f["prio"] > last["prio"]:
                last["v"], last["label"], last["prio"] = f["v"], f["label"], f["prio"]
            continue
        out.append(dict(f))
    return dict(lines=[f["v"] for f in out], labels=[f["label"] for f in out])


def grid_lines(lines, edges, hmin, hmax, spans) -> list:
    """gridLines (06-mesher.js:142-189): each interval between merged feature lines subdivided by
    the size function s(x) = min(hmax, min over refined edges of hmin + (r - 1) max(0, |x - e| - zone))
    with per-interval minimum counts from the ring and fillet spans."""
    r = GROWTH_RATIO_MAX

    def size(x):
        s = hmax
        for e in edges:
            s = min(s, hmin + (r - 1) * max(0.0, abs(x - e["v"]) - e["zone"]))
        return max(s, 1e-6)

    nmin = [1] * (len(lines) - 1)
    for sp in spans:
        ids = [q for q in range(len(lines) - 1) if lines[q] >= sp["a"] - 1e-9 and lines[q + 1] <= sp["b"] + 1e-9]
        if not ids:
            continue
        if sp.get("fillet"):
            n = _clamp(math.ceil((sp["b"] - sp["a"]) / (FILLET_COL_MIN_FRACTION * hmin)), sp.get("min") or MIN_ELEMS_ACROSS_RING,
                       MIN_ELEMS_ACROSS_FILLET)
        else:
            n = MIN_ELEMS_ACROSS_RING
        need = math.ceil(n / len(ids))
        for q in ids:
            nmin[q] = max(nmin[q], need)
    out = [lines[0]]
    M = SIZE_SAMPLES
    cum = [0.0] * (M + 1)
    for q in range(len(lines) - 1):
        a, b = lines[q], lines[q + 1]
        L = b - a
        cum[0] = 0.0
        prev = 1 / size(a)
        for m in range(1, M + 1):
            x = b if m == M else a + L * m / M
            cur = 1 / size(x)
            cum[m] = cum[m - 1] + 0.5 * (prev + cur) * L / M
            prev = cur
        I = cum[M]
        n = max(nmin[q], math.ceil(I - 1e-6), 1)
        m = 0
        for p in range(1, n):
            target = I * p / n
            while m < M and cum[m + 1] < target:
                m += 1
            t = (target - cum[m]) / max(cum[m + 1] - cum[m], 1e-300)
            out.append(a + L * (m + t) / M)
        out.append(b)
    return out


def axis_features(g: dict, axis: str) -> dict:
    """axisFeatures (06-mesher.js:196-248): feature lines, refined die and chiplet edges, ring,
    underfill and wafer underfill fillet spans, and the lid foot or stiffener ring edges."""
    sb = g["substrate"]
    lo, hi = (sb["x0"], sb["x1"]) if axis == "x" else (sb["y0"], sb["y1"])
    k0, k1 = ("x0", "x1") if axis == "x" else ("y0", "y1")
    feats = [dict(v=lo, prio=3, label="substrate edge"), dict(v=hi, prio=3, label="substrate edge")]
    edges, spans, ring_edges = [], [], []

    def add(v, prio, label):
        if lo + 1e-12 < v < hi - 1e-12:
            feats.append(dict(v=v, prio=prio, label=label))

    for d in g["dies"]:
        add(d["rect"][k0], 2, d["name"] + " edge")
        add(d["rect"][k1], 2, d["name"] + " edge")
        edges.append(dict(v=d["rect"][k0], zone=REFINE_ZONE_FACTOR * d["t"]))
        edges.append(dict(v=d["rect"][k1], zone=REFINE_ZONE_FACTOR * d["t"]))
        fa, fb = d["rect"][k0] - g["uf"]["Wf"], d["rect"][k1] + g["uf"]["Wf"]
        add(fa, 1, d["name"] + " fillet")
        add(fb, 1, d["name"] + " fillet")
        spans.append(dict(a=max(lo, fa), b=d["rect"][k0], fillet=True))
        spans.append(dict(a=d["rect"][k1], b=min(hi, fb), fillet=True))
        if d["field"]:
            add(d["field"][k0], 1, d["name"] + " bump field")
            add(d["field"][k1], 1, d["name"] + " bump field")
        if d["inner"]:
            add(d["inner"][k0], 1, d["name"] + " bump ring")
            add(d["inner"][k1], 1, d["name"] + " bump ring")
        if d["kind"] != "module":
            continue
        # chiplet edges refine like die edges; the wafer underfill fillet gets its own columns, clipped at
        # the base edge (the DDI microbump fields are not grid lines: cells take their area overlap)
        for c in d["chiplets"]:
            add(c["rect"][k0], 2, c["name"] + " edge")
            add(c["rect"][k1], 2, c["name"] + " edge")
            edges.append(dict(v=c["rect"][k0], zone=REFINE_ZONE_FACTOR * c["t"]))
            edges.append(dict(v=c["rect"][k1], zone=REFINE_ZONE_FACTOR * c["t"]))
            if not g["wcuf"]:
                continue
            wa = max(d["rect"][k0], c["rect"][k0] - g["wcuf"]["Wf"])
            wb = min(d["rect"][k1], c["rect"][k1] + g["wcuf"]["Wf"])
            add(wa, 1, c["name"] + " wCUF fillet")
            add(wb, 1, c["name"] + " wCUF fillet")
            if c["rect"][k0] - wa > 1e-9:
                spans.append(dict(a=wa, b=c["rect"][k0], fillet=True, min=1))
            if wb - c["rect"][k1] > 1e-9:
                spans.append(dict(a=c["rect"][k1], b=wb, fillet=True, min=1))
    ring = g["lid"] or g["stiff"]
    if ring:
        what = "lid" if g["lid"] else "stiffener"
        add(ring["outer"][k0], 2, what + " outer")
        add(ring["outer"][k1], 2, what + " outer")
        add(ring["inner"][k0], 2, what + " inner")
        add(ring["inner"][k1], 2, what + " inner")
        spans.append(dict(a=ring["outer"][k0], b=ring["inner"][k0]))
        spans.append(dict(a=ring["inner"][k1], b=ring["outer"][k1]))
        zone = RING_EDGE_ZONE * (g["lid"]["footH"] if g["lid"] else g["stiff"]["zTop"] - g["stiff"]["zAdhTop"])
        for v in (ring["outer"][k0], ring["inner"][k0], ring["inner"][k1], ring["outer"][k1]):
            ring_edges.append(dict(v=v, zone=zone))
    return dict(feats=feats, edges=edges, spans=spans, ringEdges=ring_edges)


# ---- z planes ------------------------------------------------------------------------------

def z_planes(g: dict) -> dict:
    """zPlanes (06-mesher.js:253-305): merged structural planes (module base tops, chiplet bottoms
    and wafer underfill fillet tops included), then element
    layers per band (die bands except slivers and the lid plate start at half the preset minimum,
    every region then gets at least the preset minimum, each extra layer to the band of the
    region with the thickest elements; substrate bands keep one layer)."""
    pl = []
    sp = g["sub"]["planes"]
    for i, z in enumerate(sp):
        pl.append(dict(v=z, label="substrate bottom" if i == 0 else ("substrate top" if i == len(sp) - 1 else "substrate band"), prio=3))
    pl.append(dict(v=g["zaf"], label="die active face", prio=2))
    Hf = g["uf"]["Hf"]
    for d in g["dies"]:
        pl.append(dict(v=d["ztop"], label=d["name"] + " top", prio=2))
        if 0 < Hf < 1:
            pl.append(dict(v=g["zaf"] + Hf * d["t"], label=d["name"] + " fillet top", prio=1))
    wc = g["wcuf"]
    for m in g["modules"]:
        pl.append(dict(v=m["zBaseTop"], label=m["name"] + " base top", prio=2))
        pl.append(dict(v=m["zDdiTop"], label=m["name"] + " chiplet bottom", prio=2))
        if wc and 0 < wc["Hf"] < 1:
            pl.append(dict(v=m["zDdiTop"] + wc["Hf"] * g["stack"]["chipletT"], label=m["name"] + " wCUF fillet top", prio=1))
    lid, stiff = g["lid"], g["stiff"]
    if lid:
        pl += [dict(v=lid["zAdhTop"], label="lid adhesive top", prio=2), dict(v=lid["zLidBot"], label="lid underside", prio=2),
               dict(v=lid["zLidTop"], label="lid top", prio=2)]
    if stiff:
        pl += [dict(v=stiff["zAdhTop"], label="stiffener adhesive top", prio=2), dict(v=stiff["zTop"], label="stiffener top", prio=2)]
    merged = merge_features(pl, PLANE_MERGE_TOL)
    base = merged["lines"]
    nmin = g["layers"]
    nstart = math.ceil(nmin / 2)
    nsub = []
    for b in range(len(base) - 1):
        za, zb = base[b], base[b + 1]
        zc = 0.5 * (za + zb)
        n = 1
        if zb > g["zt"] + 1e-9:
            t_die = math.inf
            for d in g["dies"]:
                if g["zaf"] < zc < d["ztop"]:
                    t_die = min(t_die, d["t"])
            if math.isfinite(t_die) and zb - za >= SLIVER_FRACTION * t_die:
                n = nstart
            if lid and lid["zLidBot"] < zc < lid["zLidTop"]:
                n = nstart
        nsub.append(n)
    regions = [(g["zt"], g["zaf"])]
    for d in g["dies"]:
        regions.append((g["zaf"], d["ztop"]))
        if Hf > 0:
            regions.append((g["zaf"], g["zaf"] + min(1, Hf) * d["t"]))
    # stacked modules: the base, the DDI gap, the chiplets and mold, the wafer underfill fillet
    for m in g["modules"]:
        regions += [(g["zaf"], m["zBaseTop"]), (m["zBaseTop"], m["zDdiTop"]), (m["zDdiTop"], m["ztop"])]
        if wc and wc["Hf"] > 0:
            regions.append((m["zDdiTop"], m["zDdiTop"] + min(1, wc["Hf"]) * g["stack"]["chipletT"]))
    if lid:
        regions += [(g["zt"], lid["zAdhTop"]), (lid["zAdhTop"], lid["zLidBot"]), (lid["zLidBot"], lid["zLidTop"])]
    if stiff:
        regions += [(g["zt"], stiff["zAdhTop"]), (stiff["zAdhTop"], stiff["zTop"])]
    for za, zb in regions:
        ids = [b for b in range(len(base) - 1) if za < 0.5 * (base[b] + base[b + 1]) < zb]
        if not ids:
            continue
        total = sum(nsub[b] for b in ids)
        while total < nmin:
            best = ids[0]
            for b in ids:
                if (base[b + 1] - base[b]) / nsub[b] > (base[best + 1] - base[best]) / nsub[best]:
                    best = b
            nsub[best] += 1
            total += 1
    zs, band = [base[0]], []
    for b in range(len(base) - 1):
        for s in range(1, nsub[b] + 1):
            zs.append(base[b] + (base[b + 1] - base[b]) * s / nsub[b])
            band.append(b)
    return dict(zs=zs, layerBand=band, basePlanes=base, baseLabels=merged["labels"])


# ---- groups and cell assignment --------------------------------------------------------------

def package_groups(g: dict) -> dict:
    """packageGroups (06-mesher.js:310-345): group index per role. Stacked modules add, per
    module, its chiplets, its Si base and the TSV Cu, then the DDI microbumps, the wafer underfill
    and the wafer mold (G['chip'][mi][ci], G['base'][mi], G['tsv'][mi], G['ddi'], G['wcuf'],
    G['mold'])."""
    G, names = {}, []

    def add(key, name):
        G[key] = len(names)
        names.append(name)

    add("sub", "Substrate"); add("solder", "Solder phase"); add("uf", "Underfill")
    G["die"] = []
    for i, d in enumerate(g["monoDies"]):
        G["die"].append(len(names))
        names.append(d["name"])
    if g["lid"]:
        add("tim", "TIM1"); add("lid", "Lid"); add("lidadh", "Lid adhesive")
    if g["stiff"]:
        add("stiff", "Stiffener"); add("stiffadh", "Stiffener adhesive")
    if g["modules"]:
        G["chip"], G["base"], G["tsv"] = [], [], []
        for m in g["modules"]:
            G["chip"].append([])
            for c in m["chiplets"]:
                G["chip"][-1].append(len(names))
                names.append(c["name"])
            G["base"].append(len(names))
            names.append(m["name"] + " Si base")
            G["tsv"].append(None)
            if m["tsv"] > 0:
                G["tsv"][-1] = len(names)
                names.append(m["name"] + " TSV Cu")
        add("ddi", "DDI microbumps")
        if g["wcuf"]:
            add("wcuf", "Wafer underfill")
        add("mold", "Wafer mold")
    return dict(G=G, names=names)


def _fill_fraction(hs, z_base, z0, z1) -> float:
    """fillFraction (06-mesher.js:325-329)."""
    f = 0.0
    for h in hs:
        f += _clamp((z_base + h - z0) / (z1 - z0), 0.0, 1.0)
    return f / len(hs)


def wcuf_height(g, m, x, y):
    """wcufHeight (05-geometry.js:250-253): the wafer underfill fillet height above the chiplet
    bottom at (x, y) on module m outside its chiplets (the wedge rule around the chiplets, within
    the base footprint), and whether (x, y) is in a fillet footprint."""
    if not g["wcuf"] or not _point_in_rect(m["rect"], x, y):
        return 0.0, False
    return wedge_height(m["chiplets"], g["wcuf"]["Wf"], g["wcuf"]["Hf"], x, y)


def chiplet_at(m, x, y):
    """chipletAt (05-geometry.js:262-265): the chiplet of module m whose footprint strictly holds (x, y)."""
    for c in m["chiplets"]:
        r = c["rect"]
        if r["x0"] < x < r["x1"] and r["y0"] < y < r["y1"]:
            return c
    return None


def _module_cell(g, G, d, chip, fbd, wc_in, hsw, z, z0, z1, put):
    """makePackageAssign's module branch (06-mesher.js:402-428) for a cell above the active face:
    the Si base (with the TSV Cu superposed by its fraction), the DDI gap (microbump columns
    superposed on the fill under a chiplet; wafer underfill fillet or mold between chiplets), the
    chiplet layer (chiplet, or the fillet wedge and mold by their volume fractions), the TIM above."""
    mi = d["modIndex"]
    if z < d["zBaseTop"]:
        if d["tsv"] > 0:
            put(0, G["base"][mi], PART["BASE_SI"], 1 - d["tsv"])
            put(1, G["tsv"][mi], PART["TSV"], d["tsv"])
        else:
            put(0, G["base"][mi], PART["BASE_SI"], 1.0)
    elif z < d["zDdiTop"]:
        fill = G["wcuf"] if "wcuf" in G else G["mold"]
        if chip:
            if fbd > 1e-12:
                put(0, G["ddi"], PART["DDI_SOLDER"], fbd)
                put(1, fill, PART["DDI_FILL"], 1 - fbd)
            else:
                put(0, fill, PART["DDI_FILL"], 1.0)
        elif wc_in:
            put(0, G["wcuf"], PART["WCUF_FILLET"], 1.0)
        else:
            put(0, G["mold"], PART["MOLD"], 1.0)
    elif z < d["ztop"]:
        if chip:
            put(0, G["chip"][mi][chip["index"]], PART["CHIPLET"], 1.0)
            return
        if wc_in:
            f = _fill_fraction(hsw, d["zDdiTop"], z0, z1)
            if f > 1 - FILLET_FILL_MIN:
                put(0, G["wcuf"], PART["WCUF_FILLET"], 1.0)
                return
            if f >= FILLET_FILL_MIN:
                put(0, G["wcuf"], PART["WCUF_FILLET"], f)
                put(1, G["mold"], PART["MOLD"], 1 - f)
                return
        put(0, G["mold"], PART["MOLD"], 1.0)
    elif g["lid"] and z < g["lid"]["zLidBot"]:
        put(0, G["tim"], PART["TIM"], 1.0)


def package_cells(g: dict, xs, ys, zs, G: dict):
    """makePackageAssign (06-mesher.js:344-453), evaluated for every cell:
    per-cell phase arrays (group, part, scale; two slots per cell, -1 = none) in the cell order of
    buildStructuredMesh. Column descriptors first (die under the centroid, bump fraction, fillet
    footprint and surface samples, lid and stiffener footprints), then each layer of the column."""
    nx, ny, nz = len(xs), len(ys), len(zs)
    ncy, ncz = ny - 1, nz - 1
    grp = np.full((nx - 1, ncy, ncz, 2), -1, np.int32)
    prt = np.full((nx - 1, ncy, ncz, 2), -1, np.int32)
    scl = np.zeros((nx - 1, ncy, ncz, 2), np.float64)
    zc = [0.5 * (zs[k] + zs[k + 1]) for k in range(ncz)]
    zt, zaf = g["zt"], g["zaf"]
    lid, stiff = g["lid"], g["stiff"]
    S = FILLET_FILL_SAMPLES
    ksub = [k for k in range(ncz) if zc[k] < zt]

    def put(i, j, k, q, group, part, scale):
        grp[i, j, k, q] = group; prt[i, j, k, q] = part; scl[i, j, k, q] = scale

    for i in range(nx - 1):
        for j in range(ncy):
            xc, yc = 0.5 * (xs[i] + xs[i + 1]), 0.5 * (ys[j] + ys[j + 1])
            cell = dict(x0=xs[i], x1=xs[i + 1], y0=ys[j], y1=ys[j + 1])
            die = die_at(g, xc, yc)
            fb = cell_bump_fraction(die, cell) if die else 0.0
            fil_in, hs = False, None
            if not die:
                _, fil_in = wedge_height(g["dies"], g["uf"]["Wf"], g["uf"]["Hf"], xc, yc)
                if fil_in:
                    hs = [wedge_height(g["dies"], g["uf"]["Wf"], g["uf"]["Hf"],
                                       xs[i] + (xs[i + 1] - xs[i]) * (a + 0.5) / S, ys[j] + (ys[j + 1] - ys[j]) * (b + 0.5) / S)[0]
                          for a in range(S) for b in range(S)]
            chip, fbd, wc_in, hsw = None, 0.0, False, None
            if die and die["kind"] == "module":
                chip = chiplet_at(die, xc, yc)
                fbd = cell_bump_fraction(chip, cell) if chip else 0.0
                if not chip:
                    _, wc_in = wcuf_height(g, die, xc, yc)
                    if wc_in:
                        hsw = [wcuf_height(g, die, xs[i] + (xs[i + 1] - xs[i]) * (a + 0.5) / S,
                                           ys[j] + (ys[j + 1] - ys[j]) * (b + 0.5) / S)[0] for a in range(S) for b in range(S)]
            lid_outer = lid_foot = ring = False
            if lid:
                lid_outer = _point_in_rect(lid["outer"], xc, yc)
                lid_foot = lid_outer and not _point_in_rect(lid["inner"], xc, yc)
            if stiff:
                ring = _point_in_rect(stiff["outer"], xc, yc) and not _point_in_rect(stiff["inner"], xc, yc)
            for k in ksub:
                put(i, j, k, 0, G["sub"], PART["SUB"], 1.0)
            for k in range(ncz):
                z = zc[k]
                if z < zt:
                    continue
                if lid and lid["zLidBot"] < z < lid["zLidTop"] and lid_outer:
                    put(i, j, k, 0, G["lid"], PART["LID"], 1.0)
                    continue
                if die:
                    if z < zaf:
                        if fb > 1e-12:
                            put(i, j, k, 0, G["solder"], PART["SOLDER"], fb)
                            put(i, j, k, 1, G["uf"], PART["UF_BUMP"], 1 - fb)
                        else:
                            put(i, j, k, 0, G["uf"], PART["UF_BUMP"], 1.0)
                    elif die["kind"] == "module":
                        _module_cell(g, G, die, chip, fbd, wc_in, hsw, z, zs[k], zs[k + 1], lambda *a: put(i, j, k, *a))
                    elif z < die["ztop"]:
                        put(i, j, k, 0, G["die"][die["index"]], PART["DIE"], 1.0)
                    elif lid and z < lid["zLidBot"]:
                        put(i, j, k, 0, G["tim"], PART["TIM"], 1.0)
                    continue
                if lid and lid_foot:
                    if z < lid["zAdhTop"]:
                        put(i, j, k, 0, G["lidadh"], PART["LIDADH"], 1.0)
                    elif z < lid["zLidBot"]:
                        put(i, j, k, 0, G["lid"], PART["LID"], 1.0)
                    continue
                if stiff and ring:
                    if z < stiff["zAdhTop"]:
                        put(i, j, k, 0, G["stiffadh"], PART["STIFFADH"], 1.0)
                    elif z < stiff["zTop"]:
                        put(i, j, k, 0, G["stiff"], PART["STIFF"], 1.0)
                    continue
                if fil_in:
                    if z < zaf:
                        put(i, j, k, 0, G["uf"], PART["UF_FILLET"], 1.0)
                    else:
                        f = _fill_fraction(hs, zaf, zs[k], zs[k + 1])
                        if f >= FILLET_FILL_MIN:
                            put(i, j, k, 0, G["uf"], PART["UF_FILLET"], f)
    return grp.ravel(), prt.ravel(), scl.ravel()


# ---- package mesh ------------------------------------------------------------------------------

def preset_params(cfg: dict, override: Optional[dict] = None) -> dict:
    """presetParams (06-mesher.js:455-459)."""
    name = (override or {}).get("preset") or cfg.get("mesh", {}).get("preset") or "standard"
    p = dict(MESH_PRESETS[name])
    for k in ("hmin", "hmax", "cap", "layers"):
        if override and override.get(k) is not None:
            p[k] = override[k]
    return p


def build_package_mesh(cfg: dict, override: Optional[dict] = None):
    """buildPackageMesh (06-mesher.js:468-563): the grid from the preset's
    h_min and h_max, both enlarged by sqrt(DOF / cap) x 1.03 until the DOF (3 per node) is under
    the preset cap (at most 12 times, h_min at most the preset h_max), then rebuilt with the lid
    foot or stiffener ring edges refined to the same h_min. Returns (Mesh, info)."""
    pre = preset_params(cfg, override)
    g = derive_geometry(cfg, pre["layers"])
    fx, fy = axis_features(g, "x"), axis_features(g, "y")
    mx, my = merge_features(fx["feats"], FEATURE_SNAP_TOL), merge_features(fy["feats"], FEATURE_SNAP_TOL)
    zp = z_planes(g)
    grp = package_groups(g)
    G = grp["G"]
    hmin, hmax = pre["hmin"], pre["hmax"]
    scaled = floor = False
    # with stacked modules h_min grows at most to MODULE_HMIN_PER_HEIGHT times the lowest module's height
    mod_h = [d["t"] for d in g["dies"] if d["kind"] == "module"]
    hmin_limit = max(pre["hmin"], min(pre["hmax"], MODULE_HMIN_PER_HEIGHT * min(mod_h) if mod_h else math.inf))

    def build(ring):
        xs = grid_lines(mx["lines"], fx["edges"] + fx["ringEdges"] if ring else fx["edges"], hmin, hmax, fx["spans"])
        ys = grid_lines(my["lines"], fy["edges"] + fy["ringEdges"] if ring else fy["edges"], hmin, hmax, fy["spans"])
        cg, cp, cs = package_cells(g, xs, ys, zp["zs"], G)
        return build_structured_mesh(xs, ys, zp["zs"], cg, cp, cs)

    mesh, cap_dof = None, 0
    for _ in range(CAP_MAX_ITER):
        mesh = build(False)
        cap_dof = 3 * mesh.nn
        if cap_dof <= pre["cap"] or (override and override.get("noCap")) or floor:
            break
        f = math.sqrt(cap_dof / pre["cap"]) * CAP_GROWTH_PAD
        if hmin * f >= hmin_limit:
            f = hmin_limit / hmin
            floor = True
        hmin *= f
        hmax *= f
        scaled = True
    ring_refined = len(fx["ringEdges"]) > 0
    if ring_refined:
        mesh = build(True)

    def feat_idx(lines, labels, grid):
        out = []
        for q, v in enumerate(lines):
            lab = labels[q]
            structural = lab.endswith(" edge") or lab.endswith("outer") or lab.endswith("inner")
            if not structural or "substrate" in lab:
                continue
            d = np.abs(np.asarray(grid) - v)
            best = int(np.argmin(d))
            if d[best] < 1e-9:
                out.append(best)
        return np.asarray(out, np.int32)

    mesh.featureX = feat_idx(mx["lines"], mx["labels"], mesh.xs)
    mesh.featureY = feat_idx(my["lines"], my["labels"], mesh.ys)
    sb = g["substrate"]
    mesh.constraints = constraints321(mesh, CONSTRAINT_SPAN * min(sb["x1"], sb["y1"]))
    # stacked modules are free bodies in their own process stages: a 3-2-1 support on each base bottom
    if g["modules"]:
        kb = next(k for k, z in enumerate(zp["zs"]) if abs(z - g["zaf"]) < 1e-9)
        dofs = []
        for m in g["modules"]:
            sup = module_support(mesh, m["rect"], m["cx"], m["cy"], kb)
            if sup is None:
                raise ValueError(m["name"] + ": too few mesh nodes under the module base for its support in the module stages")
            dofs += [3 * sup[0], 3 * sup[0] + 1, 3 * sup[0] + 2, 3 * sup[1] + 1, 3 * sup[1] + 2, 3 * sup[2] + 2]
        mesh.moduleConstraints = np.asarray(dofs, np.int32)
    info = dict(preset=pre["label"], hmin=hmin, hmax=hmax, cap=pre["cap"], scaled=scaled, capDof=cap_dof, capFloor=floor,
                hminLimit=hmin_limit, moduleLimited=hmin_limit < pre["hmax"],
                ringRefined=ring_refined, nx=mesh.nx, ny=mesh.ny, nz=mesh.nz, nNodes=mesh.nn, nElem=mesh.ne, nDof=3 * mesh.nn,
                layerBand=np.asarray(zp["layerBand"], np.int32), basePlanes=zp["basePlanes"], planeLabels=zp["baseLabels"],
                groups=grp["names"], geometry=g)
    return mesh, info
