"""Synthetic package models with the shapes of the tool's inputs.

A package is what the tool's JavaScript side hands to the solve path: grid
lines, a per-cell assignment of groups (``buildStructuredMesh`` input,
src/core/06-mesher.js:14), the groups' property sets per step
(``FEModel.prepareStep``, src/core/09-assembly.js:346-365) and the constraint
DOFs. The reference's verification suite builds its box models the same way
(``boxModel``, src/core/15-verify.js:11-17).

Workloads (sizes of the reference's benchmark configurations, synthetic data):

* ``box``: homogeneous or layered boxes of the verification tests.
* ``fcbga_c1``: plain FCBGA, 48x48x20 elements, substrate 35x35x1.2 mm, die
  15x15x0.775 mm, 0.08 mm bump/underfill layer with superposed solder-column
  (30 %) and underfill (70 %) phases; voids outside the die above the
  substrate; one 150 -> 25 degC step.
* ``lidded_c2``: lidded FCBGA, 160x160x32 elements, 55x55 mm 8-2-8 substrate
  in 12 layered bands, 25 mm die, TIM, Cu hat lid with adhesive foot; E and CTE
  jittered +-10 % per material (seeded).
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Callable, List, Optional

import numpy as np

from .materials import column_d, ec_d, iso_d, iso_ec, layered_section, silicon_d, substrate_row_ec, thermal_stress_const
from .mesh import PART, Mesh, build_structured_mesh, constraints321, module_support

CONSTRAINT_SPAN = 0.4   # 00-constants.js:52


@dataclass
class StepData:
    """Per-step property sets: homogeneous (D 36, s0 6) or layered (W 108, V 18)."""
    layered: np.ndarray      # (npset,) int32
    D: np.ndarray            # (npset*36,)
    s0: np.ndarray           # (npset*6,)
    W: np.ndarray            # (npset*108,)
    V: np.ndarray            # (npset*18,)
    born: np.ndarray         # (npset,) int32: thermal load on
    stage: int = 0
    # layered sets' sub-layers for the element stress histories: count per set (0 for homogeneous
    # sets), then per sub-layer in set order its z range (2), mean stiffness (36) and thermal
    # stress increment (6) of the step
    sub_n: Optional[np.ndarray] = None
    sub_z: Optional[np.ndarray] = None
    sub_D: Optional[np.ndarray] = None
    sub_s0: Optional[np.ndarray] = None


@dataclass
class Package:
    name: str
    mesh: Mesh
    group_layered: np.ndarray   # (ngroups,) int32
    group_stage: np.ndarray     # (ngroups,) int32
    group_pset: np.ndarray      # (ngroups,) property set of homogeneous groups
    sec_of_layer: np.ndarray    # (nz-1,) property set of layered groups per element layer
    npset: int
    step_fn: Callable[[float, float], StepData]
    Ta: float = 150.0
    Tb: float = 25.0
    meta: dict = field(default_factory=dict)
    # step data with named materials' moduli and expansion coefficients scaled,
    # scales {material: (E factor, CTE factor)} (applySensitivity's matE / matCTE, 14-sensitivity.js:89-110)
    material_step_fn: Optional[Callable[[dict, float, float], StepData]] = None

    def material_step(self, scales: dict, Ta: Optional[float] = None, Tb: Optional[float] = None) -> StepData:
        if self.material_step_fn is None:
            raise ValueError(f"package {self.name} has no named materials to scale")
        return self.material_step_fn(scales, self.Ta if Ta is None else Ta, self.Tb if Tb is None else Tb)

    @property
    def e_pset(self) -> np.ndarray:
        m = self.mesh
        k = m.eIJK[2::3]
        lay = self.group_layered[m.eGroup] != 0
        return np.where(lay, self.sec_of_layer[k], self.group_pset[m.eGroup]).astype(np.int32)

    def step(self, Ta: Optional[float] = None, Tb: Optional[float] = None, stage: int = 0) -> StepData:
        """prepareStep's property sets from Ta to Tb in a stage: a set's thermal load is on when one
        of its groups is born in the stage (09-assembly.js:346-365, isBorn :339)."""
        st = self.step_fn(self.Ta if Ta is None else Ta, self.Tb if Tb is None else Tb)
        st.stage = int(stage)
        if stage != 0 or np.any(self.group_stage != 0):
            born = np.zeros(self.npset, np.int32)
            k = self.mesh.eIJK[2::3]
            for g in range(len(self.group_stage)):
                if self.group_stage[g] > stage:
                    continue
                if self.group_layered[g]:
                    born[np.unique(self.sec_of_layer[k[self.mesh.eGroup == g]])] = 1
                else:
                    born[self.group_pset[g]] = 1
            st.born = born
        return st


def _homog_step(mats, Ta, Tb, npset=None, layered_fn=None) -> StepData:
    """mats: list over property sets of (D36, cte_xy, cte_z) or None for layered ones."""
    n = len(mats) if npset is None else npset
    lay = np.zeros(n, np.int32); D = np.zeros(n * 36); s0 = np.zeros(n * 6)
    W = np.zeros(n * 108); V = np.zeros(n * 18)
    sub_n = np.zeros(n, np.int32); sz, sD, sS = [], [], []
    for p, m in enumerate(mats):
        if m is None:
            lay[p] = 1
            Wp, Vp, (z, d, s) = layered_fn(p, Ta, Tb)
            W[108 * p:108 * p + 108] = Wp; V[18 * p:18 * p + 18] = Vp
            sub_n[p] = len(z) // 2; sz.append(z); sD.append(d); sS.append(s)
        else:
            Dp, axy, az = m
            D[36 * p:36 * p + 36] = Dp
            s0[6 * p:6 * p + 6] = thermal_stress_const(Dp, axy, az, Ta, Tb)
    cat = lambda a: np.concatenate(a) if a else np.zeros(0)
    return StepData(layered=lay, D=D, s0=s0, W=W, V=V, born=np.ones(n, np.int32), sub_n=sub_n, sub_z=cat(sz), sub_D=cat(sD),
                    sub_s0=cat(sS))


def linspace(a, b, n):
    """linspace of the verification suite (15-verify.js:3): n intervals, n+1 points."""
    return [a + (b - a) * i / n for i in range(n + 1)]


def box_package(xs, ys, zs, mats, assign, name="box", constraints=None, Ta=25.0, Tb=125.0) -> Package:
    """boxModel (15-verify.js:11-17): one homogeneous group per material, assign(i, j, k) -> group."""
    nx, ny, nz = len(xs), len(ys), len(zs)
    ncells = (nx - 1) * (ny - 1) * (nz - 1)
    cg = np.full(2 * ncells, -1, np.int32); cp = np.zeros(2 * ncells, np.int32); cs = np.zeros(2 * ncells)
    c = 0
    for i in range(nx - 1):
        for j in range(ny - 1):
            for k in range(nz - 1):
                cg[2 * c] = assign(i, j, k); cs[2 * c] = 1.0
                c += 1
    mesh = build_structured_mesh(xs, ys, zs, cg, cp, cs)
    a = CONSTRAINT_SPAN * min((xs[-1] - xs[0]) / 2, (ys[-1] - ys[0]) / 2)
    mesh.constraints = constraints321(mesh, a) if constraints is None else np.asarray(constraints, np.int32)
    ng = len(mats)
    return Package(name=name, mesh=mesh, group_layered=np.zeros(ng, np.int32), group_stage=np.zeros(ng, np.int32),
                   group_pset=np.arange(ng, dtype=np.int32), sec_of_layer=np.zeros(nz - 1, np.int32), npset=ng,
                   step_fn=lambda Ta_, Tb_: _homog_step(mats, Ta_, Tb_), Ta=Ta, Tb=Tb)


def _graded_lines(segments):
    out = [segments[0][0]]
    for (a, b, n) in segments:
        for q in range(1, n + 1):
            out.append(a + (b - a) * q / n)
    return np.array(out)


def fcbga_c1() -> Package:
    """Plain FP64 linear-elastic FCBGA (48x48x20 elements, voids outside the die above the substrate)."""
    xs = _graded_lines([(-17.5, -7.5, 12), (-7.5, 7.5, 24), (7.5, 17.5, 12)])
    ys = xs.copy()
    z_sub = 1.2; z_bump = 0.08; z_die = 0.775
    zs = _graded_lines([(0.0, z_sub, 10), (z_sub, z_sub + z_bump, 2), (z_sub + z_bump, z_sub + z_bump + z_die, 8)])
    nx, ny, nz = len(xs), len(ys), len(zs)
    ncy, ncz = ny - 1, nz - 1
    ncells = (nx - 1) * ncy * ncz
    cg = np.full(2 * ncells, -1, np.int32); cp = np.zeros(2 * ncells, np.int32); cs = np.zeros(2 * ncells)
    I, J, K = np.meshgrid(np.arange(nx - 1), np.arange(ncy), np.arange(ncz), indexing="ij")
    c = ((I * ncy + J) * ncz + K).ravel(); I = I.ravel(); J = J.ravel(); K = K.ravel()
    in_die = (I >= 12) & (I < 36) & (J >= 12) & (J < 36)
    sub = K < 10; bump = (K >= 10) & (K < 12); die = K >= 12
    # groups: 0 substrate, 1 solder columns, 2 underfill (bump layer), 3 die
    cg[2 * c[sub]] = 0; cp[2 * c[sub]] = PART["SUB"]; cs[2 * c[sub]] = 1.0
    b = bump & in_die
    cg[2 * c[b]] = 1; cp[2 * c[b]] = PART["SOLDER"]; cs[2 * c[b]] = 0.3
    cg[2 * c[b] + 1] = 2; cp[2 * c[b] + 1] = PART["UF_BUMP"]; cs[2 * c[b] + 1] = 0.7
    d = die & in_die
    cg[2 * c[d]] = 3; cp[2 * c[d]] = PART["DIE"]; cs[2 * c[d]] = 1.0
    mesh = build_structured_mesh(xs, ys, zs, cg, cp, cs, featureX=[12, 36], featureY=[12, 36])
    mesh.constraints = constraints321(mesh, CONSTRAINT_SPAN * min(17.5, 17.5))
    mats = [(iso_d(25000.0, 0.3), 15e-6, 15e-6),          # substrate
            (column_d(40000.0, 0.4), 22.5e-6, 22.5e-6),   # SAC solder columns (E = 40 GPa)
            (iso_d(8000.0, 0.35), 30e-6, 30e-6),          # underfill
            (iso_d(130000.0, 0.28), 2.6e-6, 2.6e-6)]      # Si die
    return Package(name="fcbga_c1", mesh=mesh, group_layered=np.zeros(4, np.int32), group_stage=np.zeros(4, np.int32),
                   group_pset=np.arange(4, dtype=np.int32), sec_of_layer=np.zeros(nz - 1, np.int32), npset=4,
                   step_fn=lambda Ta, Tb: _homog_step(mats, Ta, Tb), Ta=150.0, Tb=25.0,
                   meta=dict(workload="fcbga_c1 48x48x20", bottom_plane=0,
                             # die bump field (0.15 mm pitch over the 15 mm die), BGA (1 mm pitch) and
                             # the bump layer (mid-height, part of the solder columns)
                             die=dict(cx=0.0, cy=0.0, w=15.0, h=15.0, keepout=0.15, px=0.15, py=0.15),
                             bga=dict(sx=35.0, sy=35.0, inset=0.75, pitch=1.0),
                             bump_layer=dict(zmid=z_sub + 0.5 * z_bump, part=PART["SOLDER"])))


def _stack_8_2_8(rng_mat):
    """Bottom-up substrate rows of an 8-2-8 stack (like generateStack, src/core/02-config.js:24):
    (name, thickness)."""
    rows = [("sr", 0.020)]
    for _ in range(8):
        rows += [("diel", 0.030), ("cu", 0.015)]
    rows += [("corecu", 0.018), ("core", 0.800), ("corecu", 0.018)]
    for _ in range(8):
        rows += [("cu", 0.015), ("diel", 0.030)]
    rows += [("sr", 0.020)]
    return rows


def lidded_c2(n_inplane: int = 160, seed: int = 20261203) -> Package:
    """Mixed-precision benchmark package: lidded FCBGA, n x n x 32 elements, layered 8-2-8 substrate."""
    rng = np.random.default_rng(seed)
    names = ["sr", "diel", "cu", "corecu", "core", "solder", "uf", "die", "tim", "adh", "lid"]
    base = {  # E (MPa), nu, CTE (1/degC): database-like 25 degC constants
        "sr": (3000.0, 0.35, 50e-6), "diel": (5000.0, 0.34, 40e-6), "cu": (60000.0, 0.32, 17e-6),
        "corecu": (117000.0, 0.34, 17e-6), "core": (28000.0, 0.2, 12e-6), "solder": (40000.0, 0.4, 22.5e-6),
        "uf": (8000.0, 0.35, 30e-6), "die": (130000.0, 0.28, 2.6e-6), "tim": (10.0, 0.45, 100e-6),
        "adh": (2000.0, 0.4, 60e-6), "lid": (117000.0, 0.34, 17e-6)}
    jit = {k: (rng.uniform(0.9, 1.1), rng.uniform(0.9, 1.1)) for k in names}
    mat = {k: (base[k][0] * jit[k][0], base[k][1], base[k][2] * jit[k][1]) for k in names}
    n = n_inplane
    L = 55.0
    xs = np.array([-L / 2 + L * q / n for q in range(n + 1)])
    ys = xs.copy()
    rows = _stack_8_2_8(rng)
    zr = np.concatenate([[0.0], np.cumsum([t for _, t in rows])])
    z_sub = float(zr[-1])
    # three groups (bottom build-up, core with its Cu foils, top build-up) in 4 bands each (substrateBands, 04-homogenize.js:64-105)
    i_core = [q for q, (nm, _) in enumerate(rows) if nm == "core"][0]
    z_lo, z_hi = zr[i_core - 1], zr[i_core + 2]
    bands = []
    for (g0, g1) in [(0.0, z_lo), (z_lo, z_hi), (z_hi, z_sub)]:
        for q in range(4):
            bands.append((g0 + (g1 - g0) * q / 4, g0 + (g1 - g0) * (q + 1) / 4))
    zb = [bands[0][0]] + [b1 for (_, b1) in bands]
    t_bump, t_adh, t_die, t_tim, t_lid = 0.08, 0.10, 0.775, 0.05, 0.5
    z0 = z_sub
    zs = list(zb)
    zs += [z0 + t_bump / 2, z0 + t_bump, z0 + t_adh]                           # bump (2), adhesive top (1)
    zs += list(z0 + t_adh + (t_bump + t_die - t_adh) * np.arange(1, 8) / 7)   # die above the adhesive (7)
    zs += [z0 + t_bump + t_die + t_tim]                                       # TIM (1)
    zs += list(z0 + t_bump + t_die + t_tim + t_lid * np.arange(1, 10) / 9)    # lid plate (9)
    zs = np.array(zs)
    nz = len(zs)
    assert nz == 33, nz
    ncz = nz - 1
    nb = len(bands)
    # layers: 0..11 substrate bands, 12-13 bump, 14 adhesive top / die bottom, 15-21 die, 22 TIM, 23-31 lid
    ncells = n * n * ncz
    cg = np.full(2 * ncells, -1, np.int32); cp = np.zeros(2 * ncells, np.int32); cs = np.zeros(2 * ncells)
    I, J, K = np.meshgrid(np.arange(n), np.arange(n), np.arange(ncz), indexing="ij")
    c = ((I * n + J) * ncz + K).ravel(); I = I.ravel(); J = J.ravel(); K = K.ravel()
    d0, d1 = int(round(n * (L / 2 - 12.5) / L)), int(round(n * (L / 2 + 12.5) / L))   # die footprint cells
    m0, m1 = max(1, n * 3 // 160), n - max(1, n * 3 // 160)                            # lid outline
    fw = max(2, n * 9 // 160)                                                          # lid foot width
    in_die = (I >= d0) & (I < d1) & (J >= d0) & (J < d1)
    in_lid = (I >= m0) & (I < m1) & (J >= m0) & (J < m1)
    in_foot = in_lid & ~((I >= m0 + fw) & (I < m1 - fw) & (J >= m0 + fw) & (J < m1 - fw))
    G = dict(sub=0, solder=1, uf=2, die=3, tim=4, adh=5, lid=6)
    def put(mask, g, part, scale=1.0, q=0):
        cc = c[mask]
        cg[2 * cc + q] = g; cp[2 * cc + q] = part; cs[2 * cc + q] = scale
    put(K < nb, G["sub"], PART["SUB"])
    put((K >= 12) & (K < 14) & in_die, G["solder"], PART["SOLDER"], 0.3, 0)
    put((K >= 12) & (K < 14) & in_die, G["uf"], PART["UF_BUMP"], 0.7, 1)
    put((K == 14) & in_die, G["die"], PART["DIE"])
    put((K >= 12) & (K < 15) & in_foot, G["adh"], PART["LIDADH"])
    put((K >= 15) & (K < 22) & in_die, G["die"], PART["DIE"])
    put((K >= 15) & (K < 23) & in_foot, G["lid"], PART["LID"])
    put((K == 22) & in_die, G["tim"], PART["TIM"])
    put((K >= 23) & in_lid, G["lid"], PART["LID"])
    feat = sorted({d0, d1, m0, m1, m0 + fw, m1 - fw})
    mesh = build_structured_mesh(xs, ys, zs, cg, cp, cs, featureX=feat, featureY=feat)
    mesh.constraints = constraints321(mesh, CONSTRAINT_SPAN * L / 2)
    # property sets: 0..11 layered bands, then the homogeneous groups
    hom_names = ["solder", "uf", "die", "tim", "adh", "lid"]

    def make_step(scales, Ta, Tb):
        m = {k: (mat[k][0] * scales.get(k, (1.0, 1.0))[0], mat[k][1], mat[k][2] * scales.get(k, (1.0, 1.0))[1]) for k in names}
        band_subs = []
        for (b0, b1) in bands:
            subs = []
            for q, (nm, _) in enumerate(rows):
                a, bb = max(b0, zr[q]), min(b1, zr[q + 1])
                if bb - a > 1e-12:
                    E, nu, al = m[nm]
                    subs.append((a, bb, iso_d(E, nu), al, al))
            band_subs.append((b0, b1, subs))
        mats: List = [None] * nb
        for nm in hom_names:
            E, nu, al = m[nm]
            mats.append((column_d(E, nu) if nm == "solder" else iso_d(E, nu), al, al))

        def layered_fn(p, Ta, Tb):
            b0, b1, subs = band_subs[p]
            return layered_section(b0, b1, subs, Ta, Tb, with_subs=True)
        return _homog_step(mats, Ta, Tb, layered_fn=layered_fn)
    ng = 7
    group_layered = np.array([1, 0, 0, 0, 0, 0, 0], np.int32)
    group_pset = np.array([0, nb + 0, nb + 1, nb + 2, nb + 3, nb + 4, nb + 5], np.int32)
    sec_of_layer = np.zeros(ncz, np.int32)
    sec_of_layer[:nb] = np.arange(nb)
    return Package(name="lidded_c2", mesh=mesh, group_layered=group_layered, group_stage=np.zeros(ng, np.int32),
                   group_pset=group_pset, sec_of_layer=sec_of_layer, npset=nb + len(hom_names),
                   step_fn=lambda Ta, Tb: make_step({}, Ta, Tb), Ta=150.0, Tb=25.0, material_step_fn=make_step,
                   meta=dict(workload=f"lidded_c2 {n}x{n}x32", bottom_plane=0, seed=seed, materials=list(names),
                             die=dict(cx=0.0, cy=0.0, w=25.0, h=25.0, keepout=0.2, px=0.15, py=0.15),
                             bga=dict(sx=L, sy=L, inset=1.0, pitch=1.0),
                             bump_layer=dict(zmid=z0 + 0.5 * t_bump, part=PART["SOLDER"])))


# database-like 25 degC constants (E MPa, nu, CTE 1/degC) of the reference package's materials, by
# role: substrate row types, then the package groups
REF_PKG_MATERIALS = {
    "sr": (3000.0, 0.35, 50e-6), "diel": (5000.0, 0.34, 40e-6), "cu": (60000.0, 0.32, 17e-6), "core": (28000.0, 0.2, 12e-6),
    "solder": (40000.0, 0.4, 22.5e-6), "uf": (8000.0, 0.35, 30e-6), "die": (130000.0, 0.28, 2.6e-6), "tim": (10.0, 0.45, 100e-6),
    "lid": (117000.0, 0.34, 17e-6), "lidadh": (2000.0, 0.4, 60e-6), "stiff": (117000.0, 0.34, 17e-6), "stiffadh": (2000.0, 0.4, 60e-6),
}


# the substrate materials of the reference's default stack by database id (roles above), and the
# 25 degC expansion of (100) silicon (the reference's Si CTE formula at 25 degC: 2.553 ppm/K)
REF_PKG_MATERIAL_IDS = {"psr4000": "sr", "abf_gl": "diel", "mcl_e_795g": "core", "cu": "cu"}
SI_CTE_25C = 2.553e-6


def reference_package(preset: str = "draft", cfg: Optional[dict] = None, Ta: float = 150.0, Tb: float = 25.0,
                      homogenize: bool = False) -> Package:
    """A package on the reference's own mesh: ``buildPackageMesh`` restated (``pkgmesh``) for the
    reference's default lidded single die (``defaultConfig``) or a given configuration of
    monolithic dies, at a mesh preset (Draft 65k, Standard 314k, Fine 1.18M DOF on the default
    package). The substrate is one layered group whose element layers map to its bands (the rows
    of the band as sub-layers); solder (column phase), underfill (bump layer and fillet, the fillet
    cells scaled by their filled fraction), dies, TIM, lid and adhesive as homogeneous groups with
    database-like 25 degC constants (``REF_PKG_MATERIALS``; not the reference's temperature tables).
    With homogenize, the substrate rows follow the reference's homogenization (``substrateRowEC``:
    Cu patterns of their residual ratios in the fill dielectric, the core with its plated
    through-hole Cu) and the dies take the rotated cubic stiffness of (100) silicon (``siliconD``
    'aniso') with its 25 degC expansion."""
    from .pkgmesh import build_package_mesh, default_config
    cfg = cfg or default_config()
    mesh, info = build_package_mesh(cfg, {"preset": preset})
    g = info["geometry"]
    names = info["groups"]
    sub = g["sub"]
    bands = [(b["z0"], b["z1"]) for b in sub["bands"]]
    nb = len(bands)
    ncz = mesh.nz - 1
    sec_of_layer = np.zeros(ncz, np.int32)
    for k in range(ncz):
        zc = 0.5 * (mesh.zs[k] + mesh.zs[k + 1])
        for b, (b0, b1) in enumerate(bands):
            if b0 < zc < b1:
                sec_of_layer[k] = b
    roles = ["sub", "solder", "uf"] + ["die"] * len(g["monoDies"])
    if g["lid"]:
        roles += ["tim", "lid", "lidadh"]
    if g["stiff"]:
        roles += ["stiff", "stiffadh"]
    assert len(roles) == len(names)
    hom = roles[1:]
    rows = sub["rows"]     # bottom-up, with z ranges

    def make_step(scales, Ta_, Tb_):
        m = {k: (v[0] * scales.get(k, (1.0, 1.0))[0], v[1], v[2] * scales.get(k, (1.0, 1.0))[1]) for k, v in REF_PKG_MATERIALS.items()}
        ecs = {mid: iso_ec(m[role][0], m[role][1], m[role][2]) for mid, role in REF_PKG_MATERIAL_IDS.items()}
        band_subs = []
        for (b0, b1) in bands:
            subs = []
            for r in rows:
                a, bb = max(b0, r["z0"]), min(b1, r["z1"])
                if bb - a > 1e-12:
                    if homogenize:
                        ec = substrate_row_ec(r["row"], ecs)
                        subs.append((a, bb, ec_d(ec), ec["ax"], ec["az"]))
                    else:
                        E, nu, al = m[r["row"]["type"]]
                        subs.append((a, bb, iso_d(E, nu), al, al))
            band_subs.append((b0, b1, subs))
        mats: List = [None] * nb
        for role in hom:
            E, nu, al = m[role]
            if homogenize and role == "die":
                mats.append((silicon_d("aniso"), SI_CTE_25C, SI_CTE_25C))
            else:
                mats.append((column_d(E, nu) if role == "solder" else iso_d(E, nu), al, al))

        def layered_fn(p, Ta2, Tb2):
            b0, b1, subs = band_subs[p]
            return layered_section(b0, b1, subs, Ta2, Tb2, with_subs=True)
        return _homog_step(mats, Ta_, Tb_, layered_fn=layered_fn)

    ng = len(names)
    group_layered = np.zeros(ng, np.int32)
    group_layered[0] = 1
    group_pset = np.array([0] + [nb + q for q in range(ng - 1)], np.int32)
    d0 = g["dies"][0]
    return Package(name=f"reference_{preset}" + ("_homogenized" if homogenize else ""), mesh=mesh, group_layered=group_layered, group_stage=np.zeros(ng, np.int32),
                   group_pset=group_pset, sec_of_layer=sec_of_layer, npset=nb + ng - 1,
                   step_fn=lambda Ta_, Tb_: make_step({}, Ta_, Tb_), Ta=Ta, Tb=Tb, material_step_fn=make_step,
                   meta=dict(workload=f"reference default package, {info['preset']} mesh", bottom_plane=0, mesh_info=info,
                             materials=sorted(REF_PKG_MATERIALS),
                             die=dict(cx=d0["cx"], cy=d0["cy"], w=d0["w"], h=d0["h"], keepout=cfg["dies"][0]["bump"]["keepout"],
                                      px=d0["px"], py=d0["py"]),
                             bga=dict(sx=cfg["substrate"]["sx"], sy=cfg["substrate"]["sy"], inset=1.0, pitch=1.0),
                             bump_layer=dict(zmid=g["zt"] + 0.5 * g["so"], part=PART["SOLDER"])))


def stacked_module(n_inplane: int = 192) -> Package:
    """Stacked-module package under a thermal cycle: 45 x 45 x 1.0 mm substrate, SAC305 bump layer
    (0.08 mm, solder columns 30 % with underfill) under a 30 x 30 x 0.1 mm Si base die, a 0.03 mm
    microbump / wafer-underfill layer, four 12 x 12 x 0.6 mm chiplets (2 x 2, 2 mm apart) in wafer
    mold. The module (base die, microbumps, chiplets, mold) is born in stage -1 and stands on its own
    3-2-1 support on the base die bottom; the substrate and the bump layer are born in stage 0.
    n x n uniform in-plane cells, 15 element layers; n = 192 gives about 1.2M DOF. Solder E falls
    linearly with temperature (57.4 GPa at -40 degC, 30.0 GPa at 125 degC); the other materials are
    database-like 25 degC constants."""
    n = n_inplane
    L = 45.0
    xs = np.array([-L / 2 + L * q / n for q in range(n + 1)])
    ys = xs.copy()
    t_sub, t_bump, t_base, t_mb, t_chip = 1.0, 0.08, 0.1, 0.03, 0.6
    zs = _graded_lines([(0.0, t_sub, 6), (t_sub, t_sub + t_bump, 2), (t_sub + t_bump, t_sub + t_bump + t_base, 2),
                        (t_sub + t_bump + t_base, t_sub + t_bump + t_base + t_mb, 1),
                        (t_sub + t_bump + t_base + t_mb, t_sub + t_bump + t_base + t_mb + t_chip, 4)])
    nz = len(zs)
    ncz = nz - 1
    idx = lambda x: int(round((x + L / 2) / L * n))
    b0, b1 = idx(-15.0), idx(15.0)
    chips = [(idx(-13.0), idx(-1.0)), (idx(1.0), idx(13.0))]
    ncells = n * n * ncz
    cg = np.full(2 * ncells, -1, np.int32); cp = np.zeros(2 * ncells, np.int32); cs = np.zeros(2 * ncells)
    I, J, K = np.meshgrid(np.arange(n), np.arange(n), np.arange(ncz), indexing="ij")
    c = ((I * n + J) * ncz + K).ravel(); I = I.ravel(); J = J.ravel(); K = K.ravel()
    in_base = (I >= b0) & (I < b1) & (J >= b0) & (J < b1)
    in_chip = np.zeros_like(in_base)
    for (x0, x1) in chips:
        for (y0, y1) in chips:
            in_chip |= (I >= x0) & (I < x1) & (J >= y0) & (J < y1)
    G = dict(sub=0, solder=1, uf=2, base=3, ddi=4, fill=5, chip=6, mold=7)

    def put(mask, g, part, scale=1.0, q=0):
        cc = c[mask]
        cg[2 * cc + q] = g; cp[2 * cc + q] = part; cs[2 * cc + q] = scale
    put(K < 6, G["sub"], PART["SUB"])
    put((K >= 6) & (K < 8) & in_base, G["solder"], PART["SOLDER"], 0.3, 0)
    put((K >= 6) & (K < 8) & in_base, G["uf"], PART["UF_BUMP"], 0.7, 1)
    put((K >= 8) & (K < 10) & in_base, G["base"], PART["BASE_SI"])
    put((K == 10) & in_chip, G["ddi"], PART["DDI_SOLDER"], 0.3, 0)
    put((K == 10) & in_chip, G["fill"], PART["DDI_FILL"], 0.7, 1)
    put((K == 10) & in_base & ~in_chip, G["mold"], PART["MOLD"])
    put((K > 10) & in_chip, G["chip"], PART["CHIPLET"])
    put((K > 10) & in_base & ~in_chip, G["mold"], PART["MOLD"])
    feat = sorted({b0, b1, chips[0][0], chips[0][1], chips[1][0], chips[1][1]})
    mesh = build_structured_mesh(xs, ys, zs, cg, cp, cs, featureX=feat, featureY=feat)
    mesh.constraints = constraints321(mesh, CONSTRAINT_SPAN * L / 2)
    kb = 8   # node plane of the base die bottom
    sup = module_support(mesh, dict(x0=-15.0, x1=15.0, y0=-15.0, y1=15.0), 0.0, 0.0, kb)
    mesh.moduleConstraints = np.array([3 * sup[0], 3 * sup[0] + 1, 3 * sup[0] + 2, 3 * sup[1] + 1, 3 * sup[1] + 2, 3 * sup[2] + 2],
                                      np.int32)
    # property sets, one per group: E (MPa), nu, CTE
    const = [(iso_d(25000.0, 0.3), 15e-6), None, (iso_d(8000.0, 0.35), 30e-6), (iso_d(130000.0, 0.28), 2.6e-6),
             None, (iso_d(8000.0, 0.35), 30e-6), (iso_d(130000.0, 0.28), 2.6e-6), (iso_d(20000.0, 0.3), 10e-6)]

    def solder_E(T):   # linear E(T) of the module's SAC305 (MPa)
        return 57400.0 + (30000.0 - 57400.0) * (T + 40.0) / 165.0

    def step_fn(Ta, Tb):
        Es = solder_E(0.5 * (Ta + Tb))   # the step mean of a linear E(T)
        mats = []
        for p, m in enumerate(const):
            if m is None:
                mats.append((column_d(Es, 0.4), 22.5e-6, 22.5e-6))
            else:
                mats.append((m[0], m[1], m[1]))
        return _homog_step(mats, Ta, Tb)
    return Package(name="stacked_module", mesh=mesh, group_layered=np.zeros(8, np.int32),
                   group_stage=np.array([0, 0, 0, -1, -1, -1, -1, -1], np.int32), group_pset=np.arange(8, dtype=np.int32),
                   sec_of_layer=np.zeros(ncz, np.int32), npset=8, step_fn=step_fn, Ta=217.0, Tb=25.0,
                   meta=dict(workload=f"stacked_module {n}x{n}x{ncz}", bottom_plane=0,
                             # process: the module is stress-free at the mold cure (175 degC), attached at the
                             # solder reflow (217 degC)
                             T_module=175.0, T_attach=217.0,
                             die=dict(cx=0.0, cy=0.0, w=30.0, h=30.0, keepout=0.2, px=0.15, py=0.15),
                             bga=dict(sx=L, sy=L, inset=1.0, pitch=1.0),
                             bump_layer=dict(zmid=t_sub + 0.5 * t_bump, part=PART["SOLDER"])))


def module_path_steps(pkg: Package, max_dt: float = 30.0, temps=None):
    """The thermal path of a stacked-module package: the module alone (stage -1) from its
    stress-free temperature to the attach temperature, the whole package (stage 0) from there down to
    25 degC in steps of at most max_dt, then the two cycling branches from 25 degC through the
    cycling sample temperatures (default every 10 degC from -40 to 125 degC, with 25 and both ends)
    up to the highest and down to the lowest. Returns (steps, Tb, chain, up, down)."""
    if temps is None:
        temps = sorted(set(np.arange(-40.0, 125.0 + 1e-9, 10.0).round(9).tolist()) | {-40.0, 125.0, 25.0})
    T0, Ta = pkg.meta["T_module"], pkg.meta["T_attach"]
    steps, Tb = [pkg.step(T0, Ta, stage=-1)], [Ta]
    nch = max(1, int(np.ceil((Ta - 25.0) / max_dt - 1e-9)))
    for q in range(nch):
        a, b = Ta - (Ta - 25.0) * q / nch, Ta - (Ta - 25.0) * (q + 1) / nch
        steps.append(pkg.step(a, b)); Tb.append(b)
    chain = list(range(len(steps)))
    up, down = [], []
    for seq, br in ((sorted(t for t in temps if t > 25.0), up), (sorted((t for t in temps if t < 25.0), reverse=True), down)):
        T = 25.0
        for nxt in seq:
            br.append(len(steps)); steps.append(pkg.step(T, float(nxt))); Tb.append(float(nxt))
            T = float(nxt)
    return steps, Tb, chain, up, down


def rms_warpage(mesh: Mesh, u: np.ndarray, k: int = 0) -> float:
    """RMS of the bottom-plane z-displacement about its least-squares plane (fitPlane, src/core/01-util.js:176-190)."""
    ids = mesh.nodeId.reshape(mesh.nx, mesh.ny, mesh.nz)[:, :, k]
    X, Y = np.meshgrid(mesh.xs, mesh.ys, indexing="ij")
    ok = ids >= 0
    x = X[ok]; y = Y[ok]; w = u[3 * ids[ok] + 2]
    mx, my, mw = x.mean(), y.mean(), w.mean()
    dx, dy, dw = x - mx, y - my, w - mw
    sxx, sxy, syy, sxw, syw = (dx * dx).sum(), (dx * dy).sum(), (dy * dy).sum(), (dx * dw).sum(), (dy * dw).sum()
    det = sxx * syy - sxy * sxy
    c1 = (sxw * syy - syw * sxy) / det if abs(det) > 1e-300 else 0.0
    c2 = (syw * sxx - sxw * sxy) / det if abs(det) > 1e-300 else 0.0
    r = dw - c1 * dx - c2 * dy
    return float(np.sqrt((r * r).mean()))


def pv_warpage(mesh: Mesh, u: np.ndarray, k: int = 0) -> float:
    """Peak-to-valley of the bottom-plane z-displacement about its least-squares plane (as V5, 15-verify.js:228)."""
    ids = mesh.nodeId.reshape(mesh.nx, mesh.ny, mesh.nz)[:, :, k]
    X, Y = np.meshgrid(mesh.xs, mesh.ys, indexing="ij")
    ok = ids >= 0
    x = X[ok]; y = Y[ok]; w = u[3 * ids[ok] + 2]
    A = np.stack([np.ones_like(x), x, y], 1)
    c, *_ = np.linalg.lstsq(A, w, rcond=None)
    r = w - A @ c
    return float(r.max() - r.min())
