"""Bump submodel inputs (host side): the voxel pitch cell around one bump, its cut boundary
interpolated from the global fields, and the material tables its elements use.

The numeric engine (B-bar hexes, Anand solder Gauss points, Newton with the algorithmic
tangent, IC(0)-PCG inner solves, adaptive sub-steps) runs on the GPU behind
``tm_submodel_create`` / ``tm_submodel_step`` / ``tm_submodel_run``; this module prepares what
it reads, following (paths within the reference project):

  bump_profile        bumpProfile, src/core/04-homogenize.js:282-307
  submodel_z_planes   submodelZPlanes, src/core/13-fatigue.js:494-508
  submodel_cell       the BumpSubmodel constructor's grid and material assignment, :518-548
  boundary_nodes      _boundary's node list, :646-660
  hex_n               hexN, src/core/07-element.js:33-36
  boundary_weights    _boundary's global element and trilinear weights, :661-677
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass
from typing import Optional

import numpy as np

from . import _lib
from ._lib import check, load
from .materials import NU_MAX_GLOBAL, TGRID_N

SUB_T_AVG = 0.025       # 00-constants.js:114
SUB_MARGIN = 0.05       # 00-constants.js:115
NU_MAX_SUBMODEL = 0.49  # 00-constants.js:20
MAT = dict(SUB=0, SOLDER=1, UF=2, SI=3)
SUB_PRECONDS = dict(ic=0, line=1)    # TM_SUB_PC_IC, TM_SUB_PC_LINE
HEX_XI = (-1, 1, 1, -1, -1, 1, 1, -1)
HEX_ETA = (-1, -1, 1, 1, -1, -1, 1, 1)
HEX_ZETA = (-1, -1, -1, -1, 1, 1, 1, 1)


def bump_profile(ubm: float, sro: float, dmax: float, H: float) -> dict:
    """Solder joint as a body of revolution between the pad (z = 0) and the UBM (z = H) whose
    meridian is a circular arc of the given maximum diameter: {rt, rb, rm, zm, rho, radius_at}."""
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
        def g(r):
            return math.sqrt(max(0.0, 2 * r * db - db * db)) + math.sqrt(max(0.0, 2 * r * dt - dt * dt)) - H
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
    return dict(rt=rt, rb=rb, rm=rm, zm=zm, rho=rho, H=H, radius_at=radius_at)


def submodel_z_planes(zt: float, zaf: float, nz: int, layer_only: bool = False) -> np.ndarray:
    """z planes of the cell: substrate and die slices of SUB_MARGIN, the two SUB_T_AVG averaging
    layers at the pads and the joint between them; extra layers go to the thickest bands."""
    m, ta = (0.0 if layer_only else SUB_MARGIN), SUB_T_AVG
    bands = [[zt - m, zt, 2] if m > 0 else None, [zt, zt + ta, 3], [zt + ta, zaf - ta, 2], [zaf - ta, zaf, 3],
             [zaf, zaf + m, 2] if m > 0 else None]
    if zaf - ta <= zt + ta + 1e-9:
        bands[1][1] = 0.5 * (zt + zaf); bands[2] = None; bands[3][0] = 0.5 * (zt + zaf)
    active = [b for b in bands if b]
    total = sum(b[2] for b in active)
    while total < nz:
        best, bh = 0, -1.0
        for i, b in enumerate(active):
            h = (b[1] - b[0]) / b[2]
            if h > bh:
                bh, best = h, i
        active[best][2] += 1
        total += 1
    zs = [active[0][0]]
    for b in active:
        for k in range(1, b[2] + 1):
            zs.append(b[0] + (b[1] - b[0]) * k / b[2])
    return np.array(zs, np.float64)


def submodel_cell(site_x: float, site_y: float, px: float, py: float, nxy: int, nz: int, zt: float, zaf: float,
                  profile: dict, layer_only: bool = False):
    """Grid lines of the pitch cell and the material of every cell (SUB, SOLDER, UF, SI;
    cells in (i, j, k) order, k fastest): (xs, ys, zs, cell_mat)."""
    xs = np.array([site_x - px / 2 + px * i / nxy for i in range(nxy + 1)])
    ys = np.array([site_y - py / 2 + py * i / nxy for i in range(nxy + 1)])
    zs = submodel_z_planes(zt, zaf, nz, layer_only)
    nx, ny, nzp = len(xs), len(ys), len(zs)
    cell = np.zeros((nx - 1) * (ny - 1) * (nzp - 1), np.int32)
    q = 0
    for i in range(nx - 1):
        for j in range(ny - 1):
            for k in range(nzp - 1):
                zc = 0.5 * (zs[k] + zs[k + 1])
                if zc < zt:
                    mat = MAT["SUB"]
                elif zc > zaf:
                    mat = MAT["SI"]
                else:
                    xc = 0.5 * (xs[i] + xs[i + 1]) - site_x
                    yc = 0.5 * (ys[j] + ys[j + 1]) - site_y
                    mat = MAT["SOLDER"] if math.hypot(xc, yc) <= profile["radius_at"](zc - zt) else MAT["UF"]
                cell[q] = mat
                q += 1
    return xs, ys, zs, cell


def boundary_nodes(nx: int, ny: int, nz: int) -> np.ndarray:
    """Nodes on the six faces of a full voxel grid (every cell holds an element, so node ids are
    the mesher's (i ny + j) nz + k), ascending, with their (i, j, k)."""
    out = []
    for i in range(nx):
        for j in range(ny):
            for k in range(nz):
                if i == 0 or j == 0 or k == 0 or i == nx - 1 or j == ny - 1 or k == nz - 1:
                    out.append(((i * ny + j) * nz + k, i, j, k))
    return out


def hex_n(xi: float, eta: float, zeta: float) -> np.ndarray:
    return np.array([0.125 * (1 + HEX_XI[a] * xi) * (1 + HEX_ETA[a] * eta) * (1 + HEX_ZETA[a] * zeta) for a in range(8)])


def boundary_weights(xs, ys, zs, global_mesh) -> tuple:
    """For every boundary node of the cell: the 8 nodes of the global element containing it and
    their trilinear weights (bGlob, bW: nb x 8), from a global structured mesh given as
    (gxs, gys, gzs, node_id(i, j, k), element(i, j, k) -> (conn 8 or None))."""
    from .post import clamp, find_interval
    gxs, gys, gzs, elem_conn = global_mesh
    bn = boundary_nodes(len(xs), len(ys), len(zs))
    bGlob = np.zeros((len(bn), 8), np.int32)
    bW = np.zeros((len(bn), 8))
    for q, (_, i, j, k) in enumerate(bn):
        x, y, z = float(xs[i]), float(ys[j]), float(zs[k])
        zc = min(max(z, gzs[0] + 1e-9), gzs[-1] - 1e-9)
        gi, gj, gk = find_interval(gxs, x), find_interval(gys, y), find_interval(gzs, zc)
        conn = elem_conn(gi, gj, gk)
        nat = (clamp(2 * (x - gxs[gi]) / (gxs[gi + 1] - gxs[gi]) - 1, -1, 1),
               clamp(2 * (y - gys[gj]) / (gys[gj + 1] - gys[gj]) - 1, -1, 1),
               clamp(2 * (z - gzs[gk]) / (gzs[gk + 1] - gzs[gk]) - 1, -1, 1))
        bGlob[q] = conn
        bW[q] = hex_n(*nat)
    return bGlob, bW


@dataclass
class SubmodelSpec:
    """Everything the engine reads: cell grid and materials, the boundary's global nodes and
    weights, the global fields at the global temperatures ts (nt x nglob x 3) and at 25 degC,
    the Anand solder, and tables on the 1 degC grid (solder E/F, underfill E/F, silicon F,
    substrate-slice D (381 x 36) and F (381 x 3)); si_D the silicon stiffness."""
    xs: np.ndarray
    ys: np.ndarray
    zs: np.ndarray
    cell_mat: np.ndarray
    ts: np.ndarray
    fields: np.ndarray
    u25: np.ndarray
    bGlob: np.ndarray
    bW: np.ndarray
    anand: np.ndarray
    solder_E: np.ndarray
    solder_F: np.ndarray
    uf_E: np.ndarray
    uf_F: np.ndarray
    uf_nu: float
    si_D: np.ndarray
    si_F: np.ndarray
    sub_D: np.ndarray
    sub_F: np.ndarray
    zt: float
    zaf: float
    elastic_solder: bool = False
    nu_max: float = NU_MAX_SUBMODEL
    # homogenized-layer consistency mode (opts.uniformMaterial, 13-fatigue.js:538, 556, 711-748):
    # the bump layer as one material (solder columns with volume fraction `density`, underfill),
    # every substrate element layer from the top substrate band's section: per sub-layer its z
    # range (sec_z, nsec x 2), shell stiffness table (sec_D, nsec x 381 x 36) and thermal strain
    # table (sec_F, nsec x 381 x 3)
    uniform: bool = False
    density: float = 0.0
    nu_max_global: float = NU_MAX_GLOBAL
    sec_z: Optional[np.ndarray] = None
    sec_D: Optional[np.ndarray] = None
    sec_F: Optional[np.ndarray] = None

    @property
    def nglob(self) -> int:
        return self.u25.size // 3

    @property
    def nsec(self) -> int:
        return 0 if self.sec_z is None else int(np.asarray(self.sec_z).size // 2)

    def section_arrays(self):
        """(sec_z, sec_D, sec_F) as contiguous float64 arrays (one zero each without a section)."""
        f = lambda a: np.ascontiguousarray(np.zeros(1) if a is None else np.asarray(a).reshape(-1), np.float64)
        return f(self.sec_z), f(self.sec_D), f(self.sec_F)


def synthetic_spec(nxy: int = 16, nz: int = 14, site=(2.4, 1.2), shear: float = 2e-5, seed: int = 20261203,
                   elastic_solder: bool = False) -> SubmodelSpec:
    """A bump cell of a 0.15 mm pitch flip chip (joint 0.08 mm high, 0.09 mm UBM, 0.08 mm pad,
    0.10 mm largest diameter) cut from a synthetic global deformation: one global hex around the
    cell whose 8 nodes move with the substrate's in-plane expansion and a die-to-substrate shear
    that grows with |T - 25| (shear per degC), at the global temperatures -40, 25, 125. Materials:
    SAC305 (Anand), an underfill, isotropic silicon and a substrate slice, with E and CTE jittered
    by the seed."""
    from .materials import SAC305, anand_params_array, elastic_tables, iso_d, sac305_tables
    rng = np.random.default_rng(seed)
    zt, H = 1.2, 0.08
    zaf = zt + H
    prof = bump_profile(0.09, 0.08, 0.10, H)
    xs, ys, zs, cell = submodel_cell(site[0], site[1], 0.15, 0.15, nxy, nz, zt, zaf, prof)
    # one global element around the cell
    gxs = np.array([xs[0] - 0.05, xs[-1] + 0.05]); gys = np.array([ys[0] - 0.05, ys[-1] + 0.05])
    gzs = np.array([zs[0] - 0.05, zs[-1] + 0.05])
    gconn = [0, 4, 6, 2, 1, 5, 7, 3]           # local order of the mesher over the 2x2x2 node ids (i*2 + j)*2 + k
    bGlob, bW = boundary_weights(xs, ys, zs, (gxs, gys, gzs, lambda i, j, k: gconn))
    ts = np.array([-40.0, 25.0, 125.0])
    a_sub, a_si = 15e-6 * rng.uniform(0.9, 1.1), 2.6e-6 * rng.uniform(0.9, 1.1)
    fields = np.zeros((3, 8, 3))
    for it, T in enumerate(ts):
        dT = T - 25.0
        for i in range(2):
            for j in range(2):
                for k in range(2):
                    g = (i * 2 + j) * 2 + k
                    x, y, z = gxs[i], gys[j], gzs[k]
                    a = a_sub if k == 0 else a_si       # bottom nodes follow the substrate, top the die
                    fields[it, g] = (a * dT * x + shear * abs(dT) * (z - zt), a * dT * y, 0.5 * (a_sub + a_si) * dT * z)
    u25 = fields[1].copy()
    Et, Ft = sac305_tables()
    uf_E, uf_F = elastic_tables([-40.0, 125.0], [9000.0 * rng.uniform(0.9, 1.1), 6000.0], 30e-6)
    si_E, si_F = elastic_tables([-40.0, 125.0], [130000.0, 130000.0], 2.6e-6)
    sub_E, sub_Fs = elastic_tables([-40.0, 125.0], [26000.0, 23000.0], 15e-6)
    sub_D = np.concatenate([iso_d(float(E), 0.3, NU_MAX_SUBMODEL) for E in sub_E])
    sub_F = np.repeat(sub_Fs, 3)
    return SubmodelSpec(xs=xs, ys=ys, zs=zs, cell_mat=cell, ts=ts, fields=fields.reshape(-1), u25=u25.reshape(-1),
                        bGlob=bGlob, bW=bW, anand=anand_params_array(SAC305), solder_E=Et, solder_F=Ft,
                        uf_E=uf_E, uf_F=uf_F, uf_nu=0.35, si_D=iso_d(130000.0, 0.28, NU_MAX_SUBMODEL), si_F=si_F,
                        sub_D=sub_D, sub_F=sub_F, zt=zt, zaf=zaf, elastic_solder=elastic_solder)


def uniform_spec(spec: SubmodelSpec, density: float = 0.35, seed: int = 20261204) -> SubmodelSpec:
    """The consistency-mode variant of a spec (opts.uniformMaterial, the V7 check): the bump layer
    homogenized with solder volume fraction `density`, and a synthetic top substrate band of three
    sub-layers (a resin layer, a copper-rich layer, a resin layer) whose top is the cell's zt; the
    sub-layers' shell stiffness tables (isoD clamped at NU_MAX_GLOBAL, then sublayerShellD) and
    thermal strain tables (in-plane and through-thickness CTEs) on the 1 degC grid."""
    import dataclasses
    from .materials import NU_MAX_GLOBAL, T_STRAIN_ORIGIN, TGRID_MIN, grid_table, interp_table_linear, iso_d, sublayer_shell_d
    rng = np.random.default_rng(seed)
    zt, z0 = spec.zt, float(spec.zs[0])
    h = zt - z0
    bounds = [z0 - 0.5 * h, z0 + 0.4 * h, z0 + 0.75 * h, zt]
    layers = [(9000.0, 6000.0, 0.35, 45e-6, 60e-6), (60000.0, 52000.0, 0.33, 16e-6, 30e-6), (12000.0, 9000.0, 0.34, 35e-6, 55e-6)]
    sec_D, sec_F = [], []
    for (e_lo, e_hi, nu, a_xy, a_z) in layers:
        j = rng.uniform(0.95, 1.05)
        E_of = lambda T: j * interp_table_linear([-40.0, 125.0], [e_lo, e_hi], float(T))
        Dtab = np.concatenate([sublayer_shell_d(iso_d(E_of(TGRID_MIN + i), nu, NU_MAX_GLOBAL)) for i in range(TGRID_N)])
        Ftab = np.stack([grid_table(lambda T, a=a: a * (T - T_STRAIN_ORIGIN)) for a in (a_xy, a_xy, a_z)], axis=1).reshape(-1)
        sec_D.append(Dtab); sec_F.append(Ftab)
    sec_z = np.array([[bounds[q], bounds[q + 1]] for q in range(3)], np.float64)
    return dataclasses.replace(spec, uniform=True, density=float(density), nu_max_global=NU_MAX_GLOBAL, sec_z=sec_z,
                               sec_D=np.concatenate(sec_D), sec_F=np.concatenate(sec_F))


class DeviceSubmodel:
    """BumpSubmodel on the GPU (tm_submodel_*): step (stepTo), run, and the state readers."""

    def __init__(self, spec: SubmodelSpec):
        L = load()
        f = lambda a: np.ascontiguousarray(a, np.float64)
        i32 = lambda a: np.ascontiguousarray(a, np.int32)
        keep = [f(spec.xs), f(spec.ys), f(spec.zs), i32(spec.cell_mat), f(spec.ts), f(spec.fields), f(spec.u25),
                i32(spec.bGlob).reshape(-1), f(spec.bW).reshape(-1), f(spec.solder_E), f(spec.solder_F), f(spec.uf_E),
                f(spec.uf_F), f(spec.si_D), f(spec.si_F), f(spec.sub_D), f(spec.sub_F), *spec.section_arrays()]
        P = spec.anand
        dpp = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))
        mat = _lib.TmAnandMaterial(A=P[0], QR=P[1], xi=P[2], m=P[3], shat=P[4], n=P[5], h0=P[6], a=P[7], s0=P[8], nu=P[9],
                                   Etab=dpp(keep[9]), Ftab=dpp(keep[10]))
        ipp = lambda a: a.ctypes.data_as(C.POINTER(C.c_int32))
        sp = _lib.TmSubmodelSpec(nx=len(spec.xs), ny=len(spec.ys), nz=len(spec.zs), xs=dpp(keep[0]), ys=dpp(keep[1]), zs=dpp(keep[2]),
                                 cellMat=ipp(keep[3]), nglob=spec.nglob, nt=len(spec.ts), ts=dpp(keep[4]), fields=dpp(keep[5]),
                                 u25=dpp(keep[6]), nb=len(spec.bGlob), bGlob=ipp(keep[7]), bW=dpp(keep[8]), solder=mat,
                                 elasticSolder=int(spec.elastic_solder), ufE=dpp(keep[11]), ufF=dpp(keep[12]), ufNu=float(spec.uf_nu),
                                 siD=dpp(keep[13]), siF=dpp(keep[14]), subD=dpp(keep[15]), subF=dpp(keep[16]),
                                 nuMax=float(spec.nu_max), zt=float(spec.zt), zaf=float(spec.zaf),
                                 uniformMaterial=int(spec.uniform), density=float(spec.density),
                                 nuMaxGlobal=float(spec.nu_max_global), nsec=spec.nsec, secZ=dpp(keep[17]), secD=dpp(keep[18]),
                                 secF=dpp(keep[19]))
        h = C.c_void_p()
        check(L.tm_submodel_create(C.byref(sp), C.byref(h)))
        self.h = h
        sz = np.zeros(4, np.int64)
        check(L.tm_submodel_sizes(self.h, sz.ctypes.data_as(C.c_void_p)))
        self.nn, self.ne, self.nb, self.npoints = (int(v) for v in sz)
        self.ndof = 3 * self.nn

    def close(self):
        if getattr(self, "h", None):
            load().tm_submodel_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_precond(self, kind: str):
        """Preconditioner of the inner PCG solves: "ic" (IC(0), the reference's; the default) or
        "line" (z-line block Jacobi, one launch per apply)."""
        check(load().tm_submodel_set_precond(self.h, SUB_PRECONDS[kind]))

    def counters(self) -> dict:
        """Inner solves so far and their PCG iterations summed."""
        out = np.zeros(2, np.int64)
        check(load().tm_submodel_counters(self.h, out.ctypes.data_as(C.c_void_p)))
        return dict(solves=int(out[0]), pcg_iters=int(out[1]))

    def step(self, T, dt):
        """stepTo: (converged, newton, dMax)."""
        cv = C.c_int32(); nw = C.c_int32(); dm = C.c_double()
        check(load().tm_submodel_step(self.h, float(T), float(dt), C.byref(cv), C.byref(nw), C.byref(dm)))
        return bool(cv.value), int(nw.value), float(dm.value)

    def u(self):
        out = np.zeros(self.ndof)
        check(load().tm_submodel_get(self.h, out.ctypes.data_as(C.c_void_p), None, None))
        return out

    def points(self):
        W = np.zeros(self.npoints); E = np.zeros(self.npoints)
        check(load().tm_submodel_get(self.h, None, W.ctypes.data_as(C.c_void_p), E.ctypes.data_as(C.c_void_p)))
        return W, E

    def run(self, hist, cphi=1.0, sphi=0.0, max_snaps=0) -> dict:
        """run over a cycle history (cycle_history): the reference's result record's numbers; with
        max_snaps, the section record's stress snapshots of the last cycle (tm_submodel_run_sections):
        snaps_meta (T, t, cycle, phase) and snaps (float32, n x ne x 8 x 6)."""
        n, nc = len(hist["t"]), int(hist["cycles"])
        t = np.ascontiguousarray(hist["t"], np.float64); T = np.ascontiguousarray(hist["T"], np.float64)
        cyc = np.ascontiguousarray(hist["cycle"], np.int32)
        out = np.zeros(10); pc = np.zeros(2 * nc); loop = np.zeros(4 * n)
        vp = lambda a: a.ctypes.data_as(C.c_void_p)
        if max_snaps:
            ph = np.ascontiguousarray(hist["phase"], np.int32)
            ns = np.zeros(1, np.int32); meta = np.zeros(4 * max_snaps); sig = np.zeros(48 * self.ne * max_snaps, np.float32)
            check(load().tm_submodel_run_sections(self.h, n, vp(t), vp(T), vp(cyc), vp(ph), nc, float(cphi), float(sphi), vp(out), vp(pc),
                                                  vp(loop), int(max_snaps), vp(ns), vp(meta), vp(sig)))
        else:
            check(load().tm_submodel_run(self.h, n, vp(t), vp(T), vp(cyc), nc, float(cphi), float(sphi), vp(out), vp(pc), vp(loop)))
        keys = ["dW", "dWdie", "dWsub", "dE", "dEdie", "dEsub", "stabChange", "steps", "cutbacks", "newtonPerStep"]
        rec = {k: float(out[i]) for i, k in enumerate(keys)}
        rec["perCycle"] = pc.reshape(nc, 2); rec["loop"] = loop.reshape(n, 4)
        if max_snaps:
            k = min(int(ns[0]), max_snaps)
            rec["nsnaps"] = int(ns[0])
            rec["snaps_meta"] = meta[:4 * k].reshape(k, 4); rec["snaps"] = sig[:48 * self.ne * k].reshape(k, self.ne, 8, 6)
        return rec

    def stress_snapshot(self, T) -> np.ndarray:
        """_stressSnapshot (13-fatigue.js:965-989) of the current state: float32 (ne, 8, 6)."""
        out = np.zeros(48 * self.ne, np.float32)
        check(load().tm_submodel_stress_snapshot(self.h, float(T), out.ctypes.data_as(C.c_void_p)))
        return out.reshape(self.ne, 8, 6)


def run_batch(models, hist, cphi, sphi) -> list:
    """run of several DeviceSubmodels over one history at once (tm_submodel_run_batch: every phase
    of their Newton steps one launch over all of them): a record per model."""
    n, m, nc = len(models), len(hist["t"]), int(hist["cycles"])
    t = np.ascontiguousarray(hist["t"], np.float64); T = np.ascontiguousarray(hist["T"], np.float64)
    cyc = np.ascontiguousarray(hist["cycle"], np.int32)
    cp = np.ascontiguousarray(cphi, np.float64); sp = np.ascontiguousarray(sphi, np.float64)
    handles = (C.c_void_p * n)(*[md.h.value for md in models])
    out = np.zeros((n, 10)); pc = np.zeros((n, nc, 2)); loop = np.zeros((n, m, 4)); status = np.zeros(n, np.int32)
    vp = lambda a: a.ctypes.data_as(C.c_void_p)
    check(load().tm_submodel_run_batch(n, C.cast(handles, C.c_void_p), m, vp(t), vp(T), vp(cyc), nc, vp(cp), vp(sp), vp(out), vp(pc),
                                       vp(loop), vp(status)))
    keys = ["dW", "dWdie", "dWsub", "dE", "dEdie", "dEsub", "stabChange", "steps", "cutbacks", "newtonPerStep"]
    recs = []
    for i in range(n):
        r = {k: float(out[i, j]) for j, k in enumerate(keys)}
        r["perCycle"] = pc[i]; r["loop"] = loop[i]
        recs.append(r)
    return recs

