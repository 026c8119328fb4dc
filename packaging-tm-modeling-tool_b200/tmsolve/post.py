"""Post-processing readers of the solve path over the GPU C-ABI: JEITA warpage of the bottom
surface, BGA ball and die bump sites, and the bump-layer strain table that the joint screening
integrates.

The field values come from the GPU (``tm_sample_plane`` samples the displacement field where
it lives; ``tm_accumulate_q`` / ``tm_element_strains`` march the element DOFs of the site
elements along the thermal path); this module holds the host logic around them, which works on
a few thousand numbers: site generation, plane fit, residual range, diagonal sign, shape class.
Every function follows one reference function (paths within the reference project):

  find_interval          src/core/01-util.js:12-22
  fit_plane              src/core/01-util.js:176-190
  bump_axis              src/core/05-geometry.js:23-29
  bump_field             the site grid of bumpFieldRects, src/core/05-geometry.js:45-57
  bga_sites              src/core/05-geometry.js:172-185
  die_bump_sites         src/core/05-geometry.js:188-196
  natural_coords         src/core/12-post.js:4-11
  element_in_cell        src/core/12-post.js:19-27
  warpage_jeita          src/core/12-post.js:60-109 (samplePlane :30-38 on the GPU)
  classify_warpage_shape src/core/12-post.js:111-131
  screening_sites        src/core/13-fatigue.js:296-313
  site_elements          the site -> element lookup of siteStrainTable, 13-fatigue.js:318-331
  q_along                Analysis.qAlong, src/core/11-analysis.js:298-316 (state25 :276-281)
  site_strain_table      siteStrainTable, src/core/13-fatigue.js:318-346
  state_stride           stateSize, src/core/09-assembly.js:494-499
  states_along           StateView.state (src/core/11-analysis.js:343-375) for a set of elements
  eig_sym3, max_principal  eigSym3 / maxPrincipal, src/core/01-util.js:148-173
  joint_loads            jointLoads / bumpLoads, src/core/12-post.js:245-299
  die_surface_stress     dieSurfaceStress, src/core/12-post.js:178-243
  ddi_loads              ddiLoads, src/core/12-post.js:265-276 (jointLoads of a chiplet's microbumps)
  die_corners            dieCorners, src/core/12-post.js:316-323
  perimeter_tractions    perimeterTractions, src/core/12-post.js:349-412 (uf_tractions: ufTractions
                         :331-334; wcuf_tractions: wcufTractions :336-346)

Arithmetic is plain Python floats in the reference's order of operations, so the results are
the reference's to the last bit for the same sampled values.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import Callable, Dict, List, Optional, Sequence

import numpy as np

from .packages import StepData

# 00-constants.js:98-105
DIAG_SAMPLES = 201
SIGN_MARGINAL = 0.25
SCREEN_MAX_BUMPS = 20000
SCREEN_MAX_DDI = 5000
SCREEN_KEEP_ROWS = 3
SCREEN_CORNER_BLOCK = 10
DIE_EDGE_BAND = 0.5      # 00-constants.js:86-90
TRACTION_PATCH = 0.05    # mm: the side of a traction patch
TRACTION_SAMPLES = 3     # samples per patch side
CORNER_PATCH = 0.1
PATCH_SAMPLES = 5
GP2 = 1 / math.sqrt(3)
_HX = (-1, 1, 1, -1, -1, 1, 1, -1)
_HY = (-1, -1, 1, 1, -1, -1, 1, 1)
_HZ = (-1, -1, -1, -1, 1, 1, 1, 1)


def clamp(x: float, lo: float, hi: float) -> float:
    return lo if x < lo else (hi if x > hi else x)


def find_interval(a: Sequence[float], x: float) -> int:
    """Index i with a[i] <= x < a[i+1], clamped to [0, n-2]; a ascending."""
    n = len(a)
    if x <= a[0]:
        return 0
    if x >= a[n - 1]:
        return n - 2
    lo, hi = 0, n - 1
    while hi - lo > 1:
        mid = (lo + hi) >> 1
        if a[mid] <= x:
            lo = mid
        else:
            hi = mid
    return lo


def fit_plane(xs, ys, ws) -> tuple:
    """Least-squares plane w = c0 + c1 x + c2 y (centred normal equations): (c0, c1, c2)."""
    xs = [float(v) for v in xs]; ys = [float(v) for v in ys]; ws = [float(v) for v in ws]
    n = len(ws)
    sx = sy = sw = 0.0
    for i in range(n):
        sx += xs[i]; sy += ys[i]; sw += ws[i]
    mx, my, mw = sx / n, sy / n, sw / n
    sxx = sxy = syy = sxw = syw = 0.0
    for i in range(n):
        dx = xs[i] - mx; dy = ys[i] - my; dw = ws[i] - mw
        sxx += dx * dx; sxy += dx * dy; syy += dy * dy; sxw += dx * dw; syw += dy * dw
    det = sxx * syy - sxy * sxy
    c1 = c2 = 0.0
    if abs(det) > 1e-300:
        c1 = (sxw * syy - syw * sxy) / det
        c2 = (syw * sxx - sxw * sxy) / det
    return (mw - c1 * mx - c2 * my, c1, c2)


def bump_axis(c: float, L: float, k: float, p: float) -> dict:
    """Sites along one axis of a field of length L centred at c, inset k, pitch p."""
    span0 = L - 2 * k
    if span0 < -1e-12 or p <= 0:
        return dict(n=0, first=c, last=c)
    n = math.floor(span0 / p + 1e-9) + 1
    span = (n - 1) * p
    return dict(n=n, first=c - span / 2, last=c + span / 2)


def bump_field(cx: float, cy: float, w: float, h: float, keepout: float, px: float, py: float,
               rows: int = 1, peripheral: bool = False) -> dict:
    """Bump site grid of a w x h footprint centred at (cx, cy): {nbx, nby, bx0, by0, px, py,
    rows, peripheral} (peripheral: only the outer rows carry bumps, when the field is wide
    enough to leave an inner void)."""
    ax, ay = bump_axis(cx, w, keepout, px), bump_axis(cy, h, keepout, py)
    N = max(1, round(rows or 1))
    per = bool(peripheral and ax["n"] > 0 and ay["n"] > 0 and ax["n"] > 2 * N and ay["n"] > 2 * N)
    return dict(nbx=ax["n"], nby=ay["n"], bx0=ax["first"], by0=ay["first"], px=px, py=py, rows=N, peripheral=per)


def bga_sites(sx: float, sy: float, inset: float, pitch: float, depop: Optional[dict] = None) -> dict:
    """BGA ball sites of a substrate sx x sy centred at the origin (depop: {'on', 'sx', 'sy'}
    removes the balls of a centred rectangle) and the JEITA measuring zone."""
    ax, ay = bump_axis(0, sx, inset, pitch), bump_axis(0, sy, inset, pitch)
    xs, ys = [], []
    for i in range(ax["n"]):
        for j in range(ay["n"]):
            x = ax["first"] + i * pitch
            y = ay["first"] + j * pitch
            if depop and depop.get("on") and abs(x) < depop["sx"] / 2 and abs(y) < depop["sy"] / 2:
                continue
            xs.append(x); ys.append(y)
    return dict(x=np.array(xs, np.float64), y=np.array(ys, np.float64),
                zone=dict(x0=ax["first"], x1=ax["last"], y0=ay["first"], y1=ay["last"]), nx=ax["n"], ny=ay["n"])


def die_bump_sites(d: dict) -> dict:
    """All bump sites of a die field d = {nbx, nby, bx0, by0, px, py[, peripheral, rows]}:
    {x, y, ix, iy, row}, row = distance in rows from the field edge."""
    xs, ys, ix, iy, row = [], [], [], [], []
    for i in range(d["nbx"]):
        for j in range(d["nby"]):
            r = min(i, j, d["nbx"] - 1 - i, d["nby"] - 1 - j)
            if d.get("peripheral") and r >= d["rows"]:
                continue
            xs.append(d["bx0"] + i * d["px"]); ys.append(d["by0"] + j * d["py"])
            ix.append(i); iy.append(j); row.append(r)
    return dict(x=np.array(xs, np.float64), y=np.array(ys, np.float64), ix=np.array(ix, np.int32),
                iy=np.array(iy, np.int32), row=np.array(row, np.int32))


def screening_sites(d: dict, max_sites: Optional[int] = None) -> dict:
    """Bump sites kept for screening: all of them up to the cap, else the outer rows, the corner
    blocks and an even subsample of the rest. {sites, idx, subsampled}."""
    a = die_bump_sites(d)
    n = len(a["x"])
    cap = max_sites or SCREEN_MAX_BUMPS
    if n <= cap:
        return dict(sites=a, idx=None, subsampled=False)

    def must(q):
        cb = SCREEN_CORNER_BLOCK
        return (a["row"][q] < SCREEN_KEEP_ROWS or
                ((a["ix"][q] < cb or a["ix"][q] >= d["nbx"] - cb) and (a["iy"][q] < cb or a["iy"][q] >= d["nby"] - cb)))
    keep, rest = [], []
    for q in range(n):
        (keep if must(q) else rest).append(q)
    budget = max(0, cap - len(keep))
    stride = len(rest) / max(budget, 1)
    k = 0
    while k < budget and k * stride < len(rest):
        keep.append(rest[math.floor(k * stride)])
        k += 1
    keep.sort()
    idx = np.array(keep, np.int32)
    sites = {key: a[key][idx] for key in ("x", "y", "ix", "iy", "row")}
    return dict(sites=sites, idx=idx, subsampled=True)


def natural_coords(mesh, e: int, x: float, y: float, z: float) -> tuple:
    i, j, k = (int(v) for v in mesh.eIJK[3 * e:3 * e + 3])
    xs, ys, zs = mesh.xs, mesh.ys, mesh.zs
    return (clamp(2 * (x - xs[i]) / (xs[i + 1] - xs[i]) - 1, -1, 1),
            clamp(2 * (y - ys[j]) / (ys[j + 1] - ys[j]) - 1, -1, 1),
            clamp(2 * (z - zs[k]) / (zs[k + 1] - zs[k]) - 1, -1, 1))


def element_in_cell(mesh, i: int, j: int, k: int, part: Optional[int] = None) -> int:
    ncy, ncz = mesh.ny - 1, mesh.nz - 1
    c = (i * ncy + j) * ncz + k
    for q in range(2):
        e = int(mesh.cellElems[2 * c + q])
        if e >= 0 and (part is None or int(mesh.ePart[e]) == part):
            return e
    return -1


def site_elements(mesh, sx, sy, zmid: float, part: Optional[int]) -> tuple:
    """Element of the joint layer at mid-height zmid under every site (-1: none) and the site's
    natural coordinates in it: (elem (n,), nat (n, 3))."""
    xs, ys, zs = [float(v) for v in mesh.xs], [float(v) for v in mesh.ys], [float(v) for v in mesh.zs]
    kb = find_interval(zs, zmid)
    n = len(sx)
    elem = np.full(n, -1, np.int32)
    nat = np.zeros((n, 3))
    for q in range(n):
        x, y = float(sx[q]), float(sy[q])
        e = element_in_cell(mesh, find_interval(xs, x), find_interval(ys, y), kb, part)
        elem[q] = e
        if e >= 0:
            nat[q] = natural_coords(mesh, e, x, y, zmid)
    return elem, nat


# ---- JEITA warpage ---------------------------------------------------------------------------
def _diag(sample_pts: np.ndarray, xa, ya, xb, yb):
    """Diagonal profile from its 2 + DIAG_SAMPLES sampled values (end points first)."""
    m = DIAG_SAMPLES
    wa, wb = float(sample_pts[0]), float(sample_pts[1])
    s = np.zeros(m); rel = np.zeros(m); wv = np.zeros(m)
    mx = mn = 0.0
    L = math.hypot(xb - xa, yb - ya)
    for q in range(m):
        t = q / (m - 1)
        wv[q] = float(sample_pts[2 + q])
        s[q] = t * L
        rel[q] = wv[q] - (wa + t * (wb - wa))
        if rel[q] > mx:
            mx = float(rel[q])
        if rel[q] < mn:
            mn = float(rel[q])
    return dict(s=s, w=wv, rel=rel, max=mx, min=mn)


def _diag_points(xa, ya, xb, yb):
    m = DIAG_SAMPLES
    px, py = [xa, xb], [ya, yb]
    for q in range(m):
        t = q / (m - 1)
        px.append(xa + t * (xb - xa)); py.append(ya + t * (yb - ya))
    return px, py


def classify_warpage_shape(res, pl, mag, AB, CD) -> str:
    """'dome', 'bowl', 'ring', 'saddle' or 'flat' from the two diagonal profiles."""
    if not (mag > 0):
        return "flat"

    def prof(D):
        rel = D["rel"]; m = len(rel); ic = (m - 1) >> 1
        rc = rel[ic]
        imax = imin = 0
        for q in range(m):
            if rel[q] > rel[imax]:
                imax = q
            if rel[q] < rel[imin]:
                imin = q

        def interior(i):
            t = i / (m - 1)
            return (0.08 < t < 0.4) or (0.6 < t < 0.92)
        return dict(rc=rc, max=rel[imax], min=rel[imin], maxInterior=interior(imax), minInterior=interior(imin))
    a, c = prof(AB), prof(CD)
    up = a["rc"] > 0.1 * mag and c["rc"] > 0.1 * mag
    down = a["rc"] < -0.1 * mag and c["rc"] < -0.1 * mag
    if not up and not down:
        return "saddle"
    if up and ((a["min"] < -0.2 * mag and a["minInterior"]) or (c["min"] < -0.2 * mag and c["minInterior"])):
        return "ring"
    if down and ((a["max"] > 0.2 * mag and a["maxInterior"]) or (c["max"] > 0.2 * mag and c["maxInterior"])):
        return "ring"
    if up and a["maxInterior"] and c["maxInterior"] and a["rc"] < 0.5 * a["max"] and c["rc"] < 0.5 * c["max"]:
        return "ring"
    if down and a["minInterior"] and c["minInterior"] and a["rc"] > 0.5 * a["min"] and c["rc"] > 0.5 * c["min"]:
        return "ring"
    return "dome" if up else "bowl"


def warpage_jeita(bga: dict, sampler: Callable[[np.ndarray, np.ndarray], np.ndarray]) -> dict:
    """JEITA ED-7306 / JESD22-B112 warpage of the bottom surface over the BGA measuring zone.

    sampler(x, y) returns the bottom-plane z displacement at the points (x, y) in one call
    (``model.sample_plane(u, 0, 2, x, y)`` samples on the GPU). Returns the reference's record
    without the limit-table lookup and the contour grid: signed, mag, sign, signConf, marginal,
    shape, plane (c0, c1, c2), ballW, ballRes, diagAB, diagCD, rmin, rmax."""
    bx, by = np.asarray(bga["x"], np.float64), np.asarray(bga["y"], np.float64)
    n = len(bx)
    z = bga["zone"]
    abx, aby = _diag_points(z["x0"], z["y0"], z["x1"], z["y1"])
    cdx, cdy = _diag_points(z["x0"], z["y1"], z["x1"], z["y0"])
    # one batched sample: the balls, then diagonal AB, then diagonal CD
    px = np.concatenate([bx, np.array(abx), np.array(cdx)])
    py = np.concatenate([by, np.array(aby), np.array(cdy)])
    vals = np.asarray(sampler(px, py), np.float64)
    w = vals[:n]
    pl = fit_plane(bx, by, w)
    res = np.zeros(n)
    rmin, rmax = math.inf, -math.inf
    for q in range(n):
        r = float(w[q]) - (pl[0] + pl[1] * float(bx[q]) + pl[2] * float(by[q]))
        res[q] = r
        # Math.min / Math.max: NaN once any operand is NaN
        rmin = math.nan if (math.isnan(r) or math.isnan(rmin)) else min(rmin, r)
        rmax = math.nan if (math.isnan(r) or math.isnan(rmax)) else max(rmax, r)
    mag = rmax - rmin
    m2 = 2 + DIAG_SAMPLES
    AB = _diag(vals[n:n + m2], z["x0"], z["y0"], z["x1"], z["y1"])
    CD = _diag(vals[n + m2:], z["x0"], z["y1"], z["x1"], z["y0"])
    s = AB["max"] + AB["min"] + CD["max"] + CD["min"]
    sign = 1 if s > 0 else (-1 if s < 0 else 0)
    sign_conf = abs(s) / mag if mag > 0 else 0
    return dict(signed=sign * mag, mag=mag, sign=sign, signConf=sign_conf, marginal=sign_conf < SIGN_MARGINAL,
                shape=classify_warpage_shape(res, pl, mag, AB, CD), plane=pl, ballW=w, ballRes=res,
                diagAB=AB, diagCD=CD, rmin=rmin, rmax=rmax)


# ---- element DOF histories along the thermal path and the site strain table -------------------
@dataclass
class ThermalPath:
    """The steps of an analysis as Analysis keeps them for the stress histories: per step its
    property-set data (prepareStep's output), its end temperature Tb and its displacement
    increment du (kept as float32 by the reference, src/core/11-analysis.js:256); chain: the
    steps from the stress-free state to the as-assembled 25 degC state; up / down: the cycling
    branches from 25 degC to Tmax / Tmin."""
    steps: List[StepData]
    Tb: List[float]
    du: List[np.ndarray]
    chain: List[int]
    up: List[int] = field(default_factory=list)
    down: List[int] = field(default_factory=list)


def q_along(model, path: ThermalPath, elems, temps) -> Dict[float, np.ndarray]:
    """Element DOFs q (nel x 33) of every listed element at each of the given as-assembled
    temperatures: the 25 degC state (the chain), then both branches marched from it. All
    elements advance together, one GPU launch per step."""
    elems = np.ascontiguousarray(elems, np.int32)
    nel = len(elems)
    want = set(float(t) for t in temps)
    hi, lo = max(want), min(want)
    base = np.zeros(33 * nel)
    for k in path.chain:
        model.prepare_step(path.steps[k])
        model.accumulate_q(path.du[k], elems, base)
    out: Dict[float, np.ndarray] = {}
    if 25.0 in want:
        out[25.0] = base.reshape(nel, 33).copy()
    for br, end in ((path.up, hi), (path.down, lo)):
        if end == 25:
            continue
        st = base.copy()
        for k in br:
            model.prepare_step(path.steps[k])
            model.accumulate_q(path.du[k], elems, st)
            T = float(path.Tb[k])
            if T in want:
                out[T] = st.reshape(nel, 33).copy()
            if T == end:
                break
    return out


def site_strain_table(model, path: ThermalPath, sites: dict, temps, zmid: float, part: Optional[int]) -> np.ndarray:
    """Bump-layer total strain (engineering, xx yy zz xy yz zx) at every site for every sample
    temperature: (nsites x ntemps x 6), NaN where a site has no element of the joint layer or a
    temperature is not reached by the path."""
    mesh = model.pkg.mesh
    temps = [float(t) for t in temps]
    n, nt = len(sites["x"]), len(temps)
    out = np.full(n * nt * 6, np.nan)
    elem, nat = site_elements(mesh, sites["x"], sites["y"], zmid, part)
    have = elem >= 0
    if not have.any():
        return out
    uniq, inv = np.unique(elem[have], return_inverse=True)
    qs = q_along(model, path, uniq, temps)
    idx = np.nonzero(have)[0]
    for ti, T in enumerate(temps):
        qv = qs.get(T)
        if qv is None:
            continue
        eps = model.element_strains(elem[have], qv[inv], nat[have])
        for r, q in enumerate(idx):
            out[(q * nt + ti) * 6:(q * nt + ti) * 6 + 6] = eps[r]
    return out


# ---- element stress histories and the stress readers ------------------------------------------
def state_stride(step) -> int:
    """Doubles per element state: q (33), then per sub-layer 7 monomial stresses and the thermal
    stress (48), for the largest sub-layer count of the step's property sets."""
    ns = int(np.max(step.sub_n)) if step.sub_n is not None and len(step.sub_n) else 1
    return 33 + 48 * max(1, ns)


def states_along(model, path: ThermalPath, elems, temps, stride: int) -> Dict[float, np.ndarray]:
    """Element history states (nel x stride) at the as-assembled temperatures: the 25 degC state
    (the chain), then each branch marched from it (StateView.state); one launch per step."""
    elems = np.ascontiguousarray(elems, np.int32)
    nel = len(elems)
    want = set(float(t) for t in temps)
    hi, lo = max(want), min(want)
    base = np.zeros(stride * nel)

    def advance(k, st):
        model.prepare_step(path.steps[k])
        model.set_sublayers(path.steps[k])
        model.accumulate_state(path.du[k], elems, stride, st)
    for k in path.chain:
        advance(k, base)
    out: Dict[float, np.ndarray] = {}
    if 25.0 in want:
        out[25.0] = base.reshape(nel, stride).copy()
    for br, end in ((path.up, hi), (path.down, lo)):
        if end == 25:
            continue
        st = base.copy()
        for k in br:
            advance(k, st)
            T = float(path.Tb[k])
            if T in want:
                out[T] = st.reshape(nel, stride).copy()
            if T == end:
                break
    return out


def eig_sym3(s) -> tuple:
    """Eigenvalues, descending, of the symmetric tensor in Voigt order (xx yy zz xy yz zx)."""
    a, b, c, d, e, f = (float(v) for v in s[:6])
    p1 = d * d + e * e + f * f
    if p1 <= 1e-30 * (a * a + b * b + c * c + 1e-300):
        x, y, z = a, b, c
        if x < y:
            x, y = y, x
        if y < z:
            y, z = z, y
        if x < y:
            x, y = y, x
        return (x, y, z)
    q = (a + b + c) / 3
    p2 = (a - q) * (a - q) + (b - q) * (b - q) + (c - q) * (c - q) + 2 * p1
    p = math.sqrt(p2 / 6)
    B0, B1, B2, B3, B4, B5 = (a - q) / p, (b - q) / p, (c - q) / p, d / p, e / p, f / p
    detB = B0 * (B1 * B2 - B4 * B4) - B3 * (B3 * B2 - B4 * B5) + B5 * (B3 * B4 - B1 * B5)
    r = clamp(detB / 2, -1, 1)
    phi = math.acos(r) / 3
    e1 = q + 2 * p * math.cos(phi)
    e3 = q + 2 * p * math.cos(phi + 2 * math.pi / 3)
    return (e1, 3 * q - e1 - e3, e3)


def max_principal(s) -> float:
    return eig_sym3(s)[0]


def joint_loads(model, states: np.ndarray, state_elems, stride: int, sites: dict, zmid: float, part: Optional[int], A: float) -> dict:
    """Per-joint axial force N = szz A and shear force V = |(tyz, tzx)| A at the bump sites from the
    element states at one temperature (states[t] the state of element state_elems[t]), with the
    worst axial and shear joints and the ten largest |(N, V)|."""
    mesh = model.pkg.mesh
    n = len(sites["x"])
    N = np.full(n, np.nan); V = np.full(n, np.nan); szz = np.full(n, np.nan)
    elem, nat = site_elements(mesh, sites["x"], sites["y"], zmid, part)
    have = np.nonzero(elem >= 0)[0]
    if len(have):
        row = {int(e): t for t, e in enumerate(np.asarray(state_elems))}
        idx = np.array([row[int(elem[q])] for q in have])
        _, sig = model.state_stress(elem[have], states[idx], stride, nat[have])
        for r, q in enumerate(have):
            szz[q] = sig[r, 2]
            N[q] = sig[r, 2] * A
            V[q] = math.hypot(sig[r, 4], sig[r, 5]) * A
    worstN, worstV, iN, iV = -math.inf, -math.inf, -1, -1
    for q in range(n):
        if math.isfinite(N[q]) and abs(N[q]) > worstN:
            worstN, iN = abs(N[q]), q
        if math.isfinite(V[q]) and V[q] > worstV:
            worstV, iV = V[q], q
    order = sorted([q for q in range(n) if math.isfinite(V[q])], key=lambda q: -math.hypot(N[q], V[q]))[:10]
    return dict(N=N, V=V, szz=szz, worstN=N[iN] if iN >= 0 else math.nan, worstV=V[iV] if iV >= 0 else math.nan,
                worstNidx=iN, worstVidx=iV, worst=[dict(q=q, x=float(sites["x"][q]), y=float(sites["y"][q]), N=float(N[q]), V=float(V[q]))
                                                   for q in order], abump=A)


def plane_index(mesh, z: float) -> int:
    best, bd = 0, math.inf
    for k in range(mesh.nz):
        d = abs(float(mesh.zs[k]) - z)
        if d < bd:
            bd, best = d, k
    return best


def _gp_to_node() -> np.ndarray:
    s = math.sqrt(3)
    M = np.zeros(64)
    for n in range(8):
        N = [0.125 * (1 + _HX[g] * _HX[n] * s) * (1 + _HY[g] * _HY[n] * s) * (1 + _HZ[g] * _HZ[n] * s) for g in range(8)]
        for g in range(8):
            M[n * 8 + g] = N[g]
    return M


def die_elements(mesh, rect: dict, k_elem: int, part: Optional[int], group: int) -> list:
    """The elements of one silicon part on element layer k_elem over its footprint: (i, j, e)."""
    xs, ys = [float(v) for v in mesh.xs], [float(v) for v in mesh.ys]
    i0, i1 = find_interval(xs, rect["x0"] + 1e-9), find_interval(xs, rect["x1"] - 1e-9) + 1
    j0, j1 = find_interval(ys, rect["y0"] + 1e-9), find_interval(ys, rect["y1"] - 1e-9) + 1
    out = []
    for i in range(i0, i1):
        for j in range(j0, j1):
            e = element_in_cell(mesh, i, j, k_elem, part)
            if e >= 0 and int(mesh.eGroup[e]) == group:
                out.append((i, j, e))
    return out, (i0, i1, j0, j1)


def die_surface_stress(model, states: np.ndarray, state_elems, stride: int, rect: dict, ztop: float, zb: float, part: Optional[int],
                       group: int, which: str = "top") -> dict:
    """Nodal-averaged stress on the top or bottom face of a silicon part from its adjacent
    elements' Gauss-point stresses (extrapolated to the face nodes), the largest principal
    stress over the part's columns, its interior peak (outside DIE_EDGE_BAND), the Gauss-point
    peaks and the 100 um patch averages at the four corners and mid-edges."""
    mesh = model.pkg.mesh
    top = which == "top"
    kp = plane_index(mesh, ztop if top else zb)
    k_elem = kp - 1 if top else kp
    zeta_face = 1 if top else -1
    elems, (i0, i1, j0, j1) = die_elements(mesh, rect, k_elem, part, group)
    nxd, nyd = i1 - i0 + 1, j1 - j0 + 1
    total = np.zeros(nxd * nyd * 6); cnt = np.zeros(nxd * nyd, np.int64)
    band = DIE_EDGE_BAND
    inner = dict(x0=rect["x0"] + band, x1=rect["x1"] - band, y0=rect["y0"] + band, y1=rect["y1"] - band)
    inrect = lambda r, x, y: r["x0"] <= x <= r["x1"] and r["y0"] <= y <= r["y1"]
    gpPeak, gpPeakAll = -math.inf, -math.inf
    G2N = _gp_to_node()
    xs, ys = mesh.xs, mesh.ys
    if elems:
        row = {int(e): t for t, e in enumerate(np.asarray(state_elems))}
        E = np.repeat(np.array([e for _, _, e in elems], np.int32), 8)
        nat = np.tile(np.array([[_HX[g] * GP2, _HY[g] * GP2, _HZ[g] * GP2] for g in range(8)]), (len(elems), 1))
        _, sig = model.state_stress(E, states[np.array([row[int(e)] for e in E])], stride, nat)
        for t, (i, j, e) in enumerate(elems):
            gp = sig[8 * t:8 * t + 8]
            for g in range(8):
                sp = max_principal(gp[g])
                if _HZ[g] == zeta_face:
                    gx = 0.5 * (xs[i] + xs[i + 1]) + _HX[g] * GP2 * 0.5 * (xs[i + 1] - xs[i])
                    gy = 0.5 * (ys[j] + ys[j + 1]) + _HY[g] * GP2 * 0.5 * (ys[j + 1] - ys[j])
                    gpPeakAll = max(gpPeakAll, sp)
                    if inrect(inner, gx, gy):
                        gpPeak = max(gpPeak, sp)
            for a in range(8):
                if _HZ[a] != zeta_face:
                    continue
                gi, gj = i - i0 + (1 if _HX[a] > 0 else 0), j - j0 + (1 if _HY[a] > 0 else 0)
                o = (gi * nyd + gj) * 6
                for c in range(6):
                    v = 0.0
                    for g in range(8):
                        v += G2N[a * 8 + g] * float(gp[g, c])
                    total[o + c] += v
                cnt[gi * nyd + gj] += 1
    smax = np.full(nxd * nyd, np.nan); sxx = np.full(nxd * nyd, np.nan); syy = np.full(nxd * nyd, np.nan)
    for q in range(nxd * nyd):
        if not cnt[q]:
            continue
        tens = [total[6 * q + c] / cnt[q] for c in range(6)]
        smax[q] = max_principal(tens); sxx[q] = tens[0]; syy[q] = tens[1]
    gxs = [float(v) for v in xs[i0:i1 + 1]]; gys = [float(v) for v in ys[j0:j1 + 1]]
    peak, px, py = -math.inf, math.nan, math.nan
    for a in range(nxd):
        for b in range(nyd):
            v = smax[a * nyd + b]
            if not math.isfinite(v) or not inrect(inner, gxs[a], gys[b]):
                continue
            if v > peak:
                peak, px, py = v, gxs[a], gys[b]

    def sample_grid(x, y):
        a, b = find_interval(gxs, x), find_interval(gys, y)
        tx = (x - gxs[a]) / (gxs[a + 1] - gxs[a]); ty = (y - gys[b]) / (gys[b + 1] - gys[b])
        v00, v10 = smax[a * nyd + b], smax[(a + 1) * nyd + b]
        v01, v11 = smax[a * nyd + b + 1], smax[(a + 1) * nyd + b + 1]
        return (1 - tx) * (1 - ty) * v00 + tx * (1 - ty) * v10 + (1 - tx) * ty * v01 + tx * ty * v11

    def patch(xa, ya):
        P, m = CORNER_PATCH, PATCH_SAMPLES
        acc = 0.0
        for a in range(m):
            for b in range(m):
                acc += sample_grid(xa + P * (a + 0.5) / m, ya + P * (b + 0.5) / m)
        return acc / (m * m)
    P, r = CORNER_PATCH, rect
    corners = [(1, r["x1"], r["y0"], 1, -1), (2, r["x0"], r["y0"], -1, -1), (3, r["x0"], r["y1"], -1, 1), (4, r["x1"], r["y1"], 1, 1)]
    corner_vals = [dict(n=n, x=x, y=y, value=patch(x - P if sx > 0 else x, y - P if sy > 0 else y)) for n, x, y, sx, sy in corners]
    cx, cy = 0.5 * (r["x0"] + r["x1"]), 0.5 * (r["y0"] + r["y1"])
    mid = [dict(name="1-2", x=cx, y=r["y0"], value=patch(cx - P / 2, r["y0"])),
           dict(name="2-3", x=r["x0"], y=cy, value=patch(r["x0"], cy - P / 2)),
           dict(name="3-4", x=cx, y=r["y1"], value=patch(cx - P / 2, r["y1"] - P)),
           dict(name="4-1", x=r["x1"], y=cy, value=patch(r["x1"] - P, cy - P / 2))]
    return dict(which=which, xs=np.array(gxs), ys=np.array(gys), nx=nxd, ny=nyd, smax=smax, sxx=sxx, syy=syy, peakInterior=peak,
                peakX=px, peakY=py, gpPeakInterior=gpPeak, gpPeakAll=gpPeakAll, corners=corner_vals, midEdges=mid)



# ---- stacked-module readers and interface tractions --------------------------------------------

def ddi_loads(model, states: np.ndarray, state_elems, stride: int, g: dict, mi: int, ci: int) -> dict:
    """Per-microbump axial and shear forces of chiplet ci of module mi: joint_loads of its DDI
    sites at mid-height of the DDI gap in the microbump phase (a Cu pillar and a solder cap in
    series, so its stresses are those of both)."""
    from .mesh import PART
    m = g["modules"][mi]
    c = m["chiplets"][ci]
    r = joint_loads(model, states, state_elems, stride, die_bump_sites(c), 0.5 * (m["zBaseTop"] + m["zDdiTop"]),
                    PART["DDI_SOLDER"], c["abump"])
    r.update(module=mi, chiplet=ci)
    return r


def ddi_elements(mesh, g: dict, mi: int, ci: int) -> np.ndarray:
    """The microbump-phase elements under chiplet ci of module mi that ddi_loads reads."""
    from .mesh import PART
    m = g["modules"][mi]
    sites = die_bump_sites(m["chiplets"][ci])
    elem, _ = site_elements(mesh, sites["x"], sites["y"], 0.5 * (m["zBaseTop"] + m["zDdiTop"]), PART["DDI_SOLDER"])
    return np.unique(elem[elem >= 0])


def die_corners(r: dict) -> list:
    """The corner numbering of the tool: 1 to 4 clockwise seen from the top, from (+x, -y)."""
    return [dict(n=1, x=r["x1"], y=r["y0"], sx=1, sy=-1), dict(n=2, x=r["x0"], y=r["y0"], sx=-1, sy=-1),
            dict(n=3, x=r["x0"], y=r["y1"], sx=-1, sy=1), dict(n=4, x=r["x1"], y=r["y1"], sx=1, sy=1)]


def _perimeter_samples(mesh, r: dict, z0: float, side_parts, face_part) -> dict:
    """The sample points of perimeter_tractions with their elements: per patch (walked clockwise
    from corner 1, TRACTION_PATCH long), TRACTION_SAMPLES^2 points on the sidewall just outside
    the edge from z0 up by one patch (the first of side_parts found in the cell, else any part)
    and as many on the face just below z0, one patch deep inside the edge (face_part)."""
    step, ns, eps = TRACTION_PATCH, TRACTION_SAMPLES, 1e-6
    xs, ys, zs = [float(v) for v in mesh.xs], [float(v) for v in mesh.ys], [float(v) for v in mesh.zs]

    def elem_at(x, y, z, part):
        return element_in_cell(mesh, find_interval(xs, x), find_interval(ys, y), find_interval(zs, z), part)

    def side_elem(x, y, z):
        for p in side_parts:
            e = elem_at(x, y, z, p)
            if e >= 0:
                return e
        return elem_at(x, y, z, None)
    cs = die_corners(r)
    patches, corners, s0 = [], [0.0], 0.0
    for k, c in enumerate(cs):
        e2 = cs[(k + 1) % 4]
        nx, ny = (c["sx"] if c["sx"] == e2["sx"] else 0), (c["sy"] if c["sy"] == e2["sy"] else 0)
        L = math.hypot(e2["x"] - c["x"], e2["y"] - c["y"])
        tx, ty = (e2["x"] - c["x"]) / L, (e2["y"] - c["y"]) / L
        m = max(1, math.floor(L / step + 0.5))
        for p in range(m):
            sc = (p + 0.5) * L / m
            xc, yc = c["x"] + tx * sc, c["y"] + ty * sc
            side, face = [], []
            for a in range(ns):
                for b in range(ns):
                    ds = (a + 0.5) / ns * step - step / 2
                    x, y = xc + tx * ds, yc + ty * ds
                    zS = z0 + (b + 0.5) / ns * step
                    e = side_elem(x + nx * eps, y + ny * eps, zS)
                    if e >= 0:
                        side.append((e, x + nx * eps, y + ny * eps, zS))
                    ix, iy = x - nx * (b + 0.5) / ns * step, y - ny * (b + 0.5) / ns * step
                    e = elem_at(ix, iy, z0 - eps, face_part)
                    if e >= 0:
                        face.append((e, ix, iy, z0 - eps))
            patches.append(dict(s=s0 + sc, x=xc, y=yc, nx=nx, ny=ny, side=side, face=face))
        s0 += L
        corners.append(s0)
    return dict(patches=patches, corners=corners)


def perimeter_elements(mesh, r: dict, z0: float, side_parts, face_part) -> np.ndarray:
    """The elements that perimeter_tractions reads."""
    smp = _perimeter_samples(mesh, r, z0, side_parts, face_part)
    return np.unique(np.array([q[0] for p in smp["patches"] for q in p["side"] + p["face"]], np.int32))


def perimeter_tractions(model, states: np.ndarray, state_elems, stride: int, name: str, r: dict, z0: float, side_parts,
                        face_part) -> dict:
    """Tractions along the perimeter of rectangle r on the sidewall just outside it (t = sigma n with
    the outward normal n; peel = its normal part, shear = the rest) and on the face just below z0
    (peel szz, shear |(tyz, tzx)|), each averaged over a patch's samples, with their maxima."""
    mesh = model.pkg.mesh
    smp = _perimeter_samples(mesh, r, z0, side_parts, face_part)
    pts = [q for p in smp["patches"] for q in p["side"] + p["face"]]
    sig = np.zeros((0, 6))
    if pts:
        E = np.array([q[0] for q in pts], np.int32)
        nat = np.array([natural_coords(mesh, int(q[0]), q[1], q[2], q[3]) for q in pts])
        row = {int(e): t for t, e in enumerate(np.asarray(state_elems))}
        _, sig = model.state_stress(E, states[np.array([row[int(e)] for e in E])], stride, nat)
    out = dict(s=[], x=[], y=[], peelSide=[], shearSide=[], peelFace=[], shearFace=[])
    t = 0
    for p in smp["patches"]:
        nx, ny = p["nx"], p["ny"]
        pS = vS = pF = vF = 0.0
        for _ in p["side"]:
            sg = sig[t]; t += 1
            t0, t1, t2 = sg[0] * nx + sg[3] * ny, sg[3] * nx + sg[1] * ny, sg[5] * nx + sg[4] * ny
            tn = t0 * nx + t1 * ny
            pS += tn
            vS += math.hypot(t0 - tn * nx, t1 - tn * ny, t2)
        for _ in p["face"]:
            sf = sig[t]; t += 1
            pF += sf[2]
            vF += math.hypot(sf[4], sf[5])
        cS, cF = len(p["side"]), len(p["face"])
        out["s"].append(p["s"]); out["x"].append(p["x"]); out["y"].append(p["y"])
        out["peelSide"].append(pS / cS if cS else math.nan); out["shearSide"].append(vS / cS if cS else math.nan)
        out["peelFace"].append(pF / cF if cF else math.nan); out["shearFace"].append(vF / cF if cF else math.nan)
    mx = lambda a: max([v for v in a if math.isfinite(v)], default=-math.inf)
    res = {k: np.array(v) for k, v in out.items()}
    res.update(die=name, corners=smp["corners"], maxPeelSide=mx(out["peelSide"]), maxShearSide=mx(out["shearSide"]),
               maxPeelFace=mx(out["peelFace"]), maxShearFace=mx(out["shearFace"]))
    return res


def uf_tractions(model, states: np.ndarray, state_elems, stride: int, g: dict, die: int) -> dict:
    """Underfill tractions along the perimeter of a die (or module base) on the flip chip layer: the
    sidewall to the fillet, the active face to the underfill near the edge."""
    from .mesh import PART
    d = g["dies"][die]
    return perimeter_tractions(model, states, state_elems, stride, d["name"], d["rect"], d["zaf"], [PART["UF_FILLET"]],
                               PART["UF_BUMP"])


def wcuf_tractions(model, states: np.ndarray, state_elems, stride: int, g: dict, mi: int, ci: int) -> dict:
    """Wafer underfill (or wafer mold) tractions around chiplet ci of module mi: the chiplet
    sidewall to the fillet or mold, the chiplet's active face to the DDI fill near the edge."""
    from .mesh import PART
    m = g["modules"][mi]
    c = m["chiplets"][ci]
    r = perimeter_tractions(model, states, state_elems, stride, c["name"], c["rect"], m["zDdiTop"],
                            [PART["WCUF_FILLET"], PART["MOLD"]], PART["DDI_FILL"])
    r.update(module=mi, chiplet=ci, fill="wcuf" if g["wcuf"] else "mold")
    return r
