"""Per-step material data that the caller hands to the solver (the reference's
``FEModel.prepareStep`` inputs), for constant-property synthetic packages.

The material database and its temperature tables stay on the caller's side of
the boundary in the reference; this module restates the parts that synthetic
inputs need:

* ``orthoD`` / ``isoD`` / ``columnD`` (src/core/03-materials.js:222-266) with
  ``invDense`` (src/core/01-util.js:110-134);
* the constant-stiffness branch of ``gridStressIncrement`` (03-materials.js:394-401);
* layered sections: ``lagrange3Integrals`` and the W_j / V_j weights of
  ``buildBandSection`` / ``sectionVstep`` (src/core/04-homogenize.js:115-221)
  for sub-layers of constant properties, with ``sublayerShellD`` (:115-121);
* the 1 degC property grid and ``gridAt`` (03-materials.js:344-355) used by the
  Anand point (E(T) and the thermal strain F(T)).
"""
from __future__ import annotations

import numpy as np

NU_MAX_GLOBAL = 0.45          # 00-constants.js:19
COLUMN_INPLANE_FRACTION = 1e-3  # 00-constants.js:25
TGRID_MIN, TGRID_MAX = -80, 300
TGRID_N = TGRID_MAX - TGRID_MIN + 1
T_STRAIN_ORIGIN = 25.0


def inv_dense(A: np.ndarray) -> np.ndarray:
    """invDense (01-util.js:110-134): Gauss-Jordan with partial pivoting, same operation order."""
    A = np.asarray(A, np.float64)
    n = A.shape[0]
    M = np.zeros((n, 2 * n))
    M[:, :n] = A
    M[np.arange(n), n + np.arange(n)] = 1.0
    for c in range(n):
        p = c
        best = abs(M[c, c])
        for r in range(c + 1, n):
            v = abs(M[r, c])
            if v > best:
                best, p = v, r
        if best == 0:
            raise ValueError("singular matrix in invDense")
        if p != c:
            M[[c, p]] = M[[p, c]]
        inv = 1.0 / M[c, c]
        M[c] = M[c] * inv
        for r in range(n):
            if r == c:
                continue
            f = M[r, c]
            if f == 0:
                continue
            M[r] = M[r] - f * M[c]
    return M[:, n:].copy()


def ortho_d(Ex, Ey, Ez, Gxy, Gxz, Gyz, nuxy, nuxz, nuyz, nu_max=None) -> np.ndarray:
    """orthoD (03-materials.js:222-238): 6x6 Voigt stiffness (xx yy zz xy yz zx, engineering shear)."""
    cl = (lambda v: min(v, 0.499 if nu_max is None else nu_max))
    nxy, nxz, nyz = cl(nuxy), cl(nuxz), cl(nuyz)
    S = np.zeros((3, 3))
    S[0, 0] = 1 / Ex; S[1, 1] = 1 / Ey; S[2, 2] = 1 / Ez
    S[0, 1] = S[1, 0] = -nxy / Ex
    S[0, 2] = S[2, 0] = -nxz / Ex
    S[1, 2] = S[2, 1] = -nyz / Ey
    C = inv_dense(S)
    D = np.zeros(36)
    D[0], D[1], D[2] = C[0]
    D[6], D[7], D[8] = C[1]
    D[12], D[13], D[14] = C[2]
    D[21] = Gxy; D[28] = Gyz; D[35] = Gxz
    return D


def iso_d(E, nu, nu_max=NU_MAX_GLOBAL) -> np.ndarray:
    """isoD (03-materials.js:247-249) through isoEC (:241-244)."""
    nu_c = min(nu, 0.499 if nu_max is None else nu_max)
    G = E / (2 * (1 + nu_c))
    return ortho_d(E, E, E, G, G, G, nu_c, nu_c, nu_c, nu_max)


def iso_ec(E, nu, a) -> dict:
    """isoEC (03-materials.js:241-244): isotropic engineering constants."""
    G = E / (2 * (1 + nu))
    return dict(Ex=E, Ey=E, Ez=E, Gxy=G, Gxz=G, Gyz=G, nuxy=nu, nuxz=nu, nuyz=nu, ax=a, ay=a, az=a)


def ec_d(ec: dict, nu_max=NU_MAX_GLOBAL) -> np.ndarray:
    """orthoD of an engineering-constants record."""
    return ortho_d(ec["Ex"], ec["Ey"], ec["Ez"], ec["Gxy"], ec["Gxz"], ec["Gyz"], ec["nuxy"], ec["nuxz"], ec["nuyz"], nu_max)


def mix_cu_ec(cu: dict, d: dict, r: float, inplane_rule: str) -> dict:
    """The Cu-pattern mixing rules of a substrate row (mixCuEC, src/core/04-homogenize.js:14-27):
    a Cu phase of area fraction r beside a matrix phase, both through the row's thickness.
    Through-thickness modulus and shears: Voigt, X = r X_c + (1 - r) X_d. In-plane moduli and
    shear: Voigt for a plane layer ('plane'), the mean of Voigt and Reuss (1/X = r/X_c +
    (1 - r)/X_d) for a signal layer. Poisson ratios by the rule of mixtures; each direction's CTE
    by Turner's rule, (r E_c a_c + (1 - r) E_d a_d) / (r E_c + (1 - r) E_d) with that direction's
    moduli."""
    voigt = lambda xc, xd: r * xc + (1 - r) * xd
    reuss = lambda xc, xd: 1 / (r / xc + (1 - r) / xd)
    inpl = (lambda xc, xd: voigt(xc, xd)) if inplane_rule == "plane" else (lambda xc, xd: 0.5 * (voigt(xc, xd) + reuss(xc, xd)))
    turner = lambda Ec, ac, Ed, ad: (r * Ec * ac + (1 - r) * Ed * ad) / (r * Ec + (1 - r) * Ed)
    return dict(Ex=inpl(cu["Ex"], d["Ex"]), Ey=inpl(cu["Ey"], d["Ey"]), Ez=voigt(cu["Ez"], d["Ez"]),
                Gxy=inpl(cu["Gxy"], d["Gxy"]), Gxz=voigt(cu["Gxz"], d["Gxz"]), Gyz=voigt(cu["Gyz"], d["Gyz"]),
                nuxy=voigt(cu["nuxy"], d["nuxy"]), nuxz=voigt(cu["nuxz"], d["nuxz"]), nuyz=voigt(cu["nuyz"], d["nuyz"]),
                ax=turner(cu["Ex"], cu["ax"], d["Ex"], d["ax"]), ay=turner(cu["Ey"], cu["ay"], d["Ey"], d["ay"]),
                az=turner(cu["Ez"], cu["az"], d["Ez"], d["az"]))


def substrate_row_ec(row: dict, mats: dict) -> dict:
    """substrateRowEC (04-homogenize.js:35-54) at one temperature, with the materials' engineering
    constants given (mats: name -> record, 'cu' the pattern copper): solder resist and dielectric
    rows as their material (a dielectric with via Cu mixed by the signal rule), Cu rows as the Cu
    pattern of residual ratio r in the fill dielectric (plane or signal rule), the core with its
    plated-through-hole Cu by the plane rule."""
    cu = mats["cu"]
    t = row["type"]
    if t == "sr":
        return dict(mats[row["mat"]])
    if t == "diel":
        d = mats[row["mat"]]
        return mix_cu_ec(cu, d, row["via"], "signal") if row.get("via", 0) > 0 else dict(d)
    if t == "cu":
        return mix_cu_ec(cu, mats[row["fill"]], row["r"], "plane" if row["kind"] == "plane" else "signal")
    if t == "core":
        d = mats[row["mat"]]
        return mix_cu_ec(cu, d, row["pth"], "plane") if row.get("pth", 0) > 0 else dict(d)
    raise ValueError(f"unknown substrate row type {t!r}")


# silicon's cubic constants (MPa): the literature values of (100) silicon
SI_C11, SI_C12, SI_C44 = 165.7e3, 63.9e3, 79.6e3


def cubic_rotated_d(C11: float, C12: float, C44: float, theta: float) -> np.ndarray:
    """Stiffness of a cubic crystal rotated by theta about z (cubicRotatedD, 03-materials.js:272-294;
    theta = 45 degrees puts x along <110>, the die edges of (100) silicon): the fourth-order tensor
    C'_ijkl = R_ip R_jq R_kr R_ls C_pqrs in Voigt order (xx yy zz xy yz zx)."""
    c, s = np.cos(theta), np.sin(theta)
    R = np.array([[c, -s, 0.0], [s, c, 0.0], [0.0, 0.0, 1.0]])
    C = np.zeros((3, 3, 3, 3))
    for i in range(3):
        for k in range(3):
            C[i, i, k, k] = C11 if i == k else C12
    for i in range(3):
        for j in range(3):
            if i != j:
                C[i, j, i, j] = C[i, j, j, i] = C44
    Cr = np.einsum("ip,jq,kr,ls,pqrs->ijkl", R, R, R, R, C)
    vo = [(0, 0), (1, 1), (2, 2), (0, 1), (1, 2), (2, 0)]
    return np.array([Cr[i, j, k, l] for (i, j) in vo for (k, l) in vo])


def directional_modulus(D: np.ndarray, n) -> float:
    """Young's modulus along the unit direction n from a 6x6 stiffness (directionalModulus,
    03-materials.js:297-307): the normal strain along n under a unit uniaxial stress along n."""
    S = np.linalg.inv(np.asarray(D, np.float64).reshape(6, 6))
    n = np.asarray(n, np.float64)
    sv = np.array([n[0] * n[0], n[1] * n[1], n[2] * n[2], n[0] * n[1], n[1] * n[2], n[2] * n[0]])
    ev = S @ sv
    e = ev[0] * n[0] * n[0] + ev[1] * n[1] * n[1] + ev[2] * n[2] * n[2] + ev[3] * n[0] * n[1] + ev[4] * n[1] * n[2] + ev[5] * n[2] * n[0]
    return 1.0 / e


def silicon_d(model: str = "aniso") -> np.ndarray:
    """siliconD (03-materials.js:310-314): 'aniso' the cubic constants rotated by 45 degrees (die
    edges along <110>), 'iso' E = 130 GPa, nu = 0.28."""
    if model == "iso":
        return iso_d(130e3, 0.28)
    return cubic_rotated_d(SI_C11, SI_C12, SI_C44, np.pi / 4)


def column_d(E, nu) -> np.ndarray:
    """columnD (03-materials.js:259-266): solder phase of the bump layer as separate columns."""
    D = np.zeros(36)
    G = E / (2 * (1 + nu))
    fl = COLUMN_INPLANE_FRACTION
    D[0] = D[7] = fl * E
    D[21] = fl * G
    D[14] = E; D[28] = G; D[35] = G
    return D


def thermal_stress_const(D: np.ndarray, cte_xy: float, cte_z: float, Ta: float, Tb: float) -> np.ndarray:
    """gridStressIncrement with a constant stiffness (03-materials.js:397-400) for constant CTEs:
    s0[r] = sum_c D[r, c] (F_c(Tb) - F_c(Ta)), F(T) = alpha (T - 25)."""
    f = np.array([cte_xy * (Tb - T_STRAIN_ORIGIN) - cte_xy * (Ta - T_STRAIN_ORIGIN),
                  cte_xy * (Tb - T_STRAIN_ORIGIN) - cte_xy * (Ta - T_STRAIN_ORIGIN),
                  cte_z * (Tb - T_STRAIN_ORIGIN) - cte_z * (Ta - T_STRAIN_ORIGIN)])
    Dm = np.asarray(D).reshape(6, 6)
    return np.array([Dm[r, 0] * f[0] + Dm[r, 1] * f[1] + Dm[r, 2] * f[2] for r in range(6)])


def lagrange3_integrals(a: float, b: float):
    """lagrange3Integrals (04-homogenize.js:124-129)."""
    Im = lambda z: z * z * z / 6 - z * z / 4
    I0 = lambda z: z - z * z * z / 3
    Ip = lambda z: z * z * z / 6 + z * z / 4
    return [Im(b) - Im(a), I0(b) - I0(a), Ip(b) - Ip(a)]


def sublayer_shell_d(D: np.ndarray) -> np.ndarray:
    """sublayerShellD (04-homogenize.js:115-121): plane-stress in-plane block, uncoupled thickness modulus."""
    D = np.array(D, np.float64)
    zz = D[14]
    P = (0, 1, 3)
    for a in P:
        for b in P:
            D[a * 6 + b] -= D[a * 6 + 2] * D[2 * 6 + b] / zz
    for a in P:
        D[a * 6 + 2] = 0.0
        D[2 * 6 + a] = 0.0
    D[14] = zz
    return D


def layered_section(z0: float, z1: float, subs, Ta: float, Tb: float, plane_stress=True, with_subs=False):
    """Step weights of one layered band of constant-property sub-layers.

    subs: list of (sz0, sz1, D36, cte_xy, cte_z). Returns (W 108, V 18) as in
    buildBandSection's W_j (04-homogenize.js:172-181) averaged over the step
    (constant here) and sectionVstep (:212-221); with_subs adds the sub-layers'
    z ranges, step-mean stiffnesses and thermal stress increments (sectionSubMeanD,
    sectionSubStress, :196-204), which the element stress histories read."""
    h = z1 - z0
    W = np.zeros(108)
    V = np.zeros(18)
    sz, sD, sS = [], [], []
    for (sz0, sz1, D, axy, az) in subs:
        Dl = sublayer_shell_d(D) if plane_stress else np.asarray(D, np.float64)
        L = lagrange3_integrals(2 * (sz0 - z0) / h - 1, 2 * (sz1 - z0) / h - 1)
        s0 = thermal_stress_const(Dl, axy, az, Ta, Tb)
        for j in range(3):
            W[j * 36:(j + 1) * 36] += Dl * L[j]
            V[j * 6:(j + 1) * 6] += s0 * L[j]
        sz.append((sz0, sz1)); sD.append(Dl); sS.append(s0)
    if with_subs:
        return W, V, (np.array(sz, np.float64).reshape(-1), np.concatenate(sD), np.concatenate(sS))
    return W, V


def grid_table(fn) -> np.ndarray:
    """A property on the 1 degC grid TGRID_MIN..TGRID_MAX (03-materials.js:344, 424-433)."""
    return np.array([fn(float(TGRID_MIN + i)) for i in range(TGRID_N)], np.float64)


def grid_at(arr: np.ndarray, T: float) -> float:
    """gridAt (03-materials.js:347-355)."""
    x = T - TGRID_MIN
    if x <= 0:
        return float(arr[0])
    if x >= TGRID_N - 1:
        return float(arr[TGRID_N - 1])
    i = int(np.floor(x)); t = x - i
    return float(arr[i] + t * (arr[i + 1] - arr[i]))


def interp_table_linear(xs, ys, x):
    """interpTable with linear extrapolation (01-util.js:25-33)."""
    n = len(xs)
    if n == 1:
        return ys[0]
    if x <= xs[0]:
        i = 0
    elif x >= xs[-1]:
        i = n - 2
    else:
        lo, hi = 0, n - 1
        while hi - lo > 1:
            mid = (lo + hi) >> 1
            if xs[mid] <= x:
                lo = mid
            else:
                hi = mid
        i = lo
    t = (x - xs[i]) / (xs[i + 1] - xs[i])
    return ys[i] + t * (ys[i + 1] - ys[i])


# SAC305 of the tool's material database (src/materials-db.json, record "sac305")
SAC305 = dict(A=3501.0, QR=9320.0, xi=4.0, m=0.25, shat=30.2, n=0.01, h0=180000.0, a=1.78, s0=21.0, nu=0.4,
              E_T=[-40.0, 25.0, 75.0, 125.0], E_GPa=[57.4, 46.5, 38.2, 30.0], solidus=217.0, cte=22.5e-6)


def sac305_tables():
    """E(T) (MPa, linear table with linear extrapolation, 1 % above the solidus; 03-materials.js:88-116)
    and F(T) = alpha (T - 25) on the 1 degC grid."""
    def E(T):
        if T > SAC305["solidus"]:
            return 0.01 * interp_table_linear(SAC305["E_T"], SAC305["E_GPa"], SAC305["solidus"]) * 1000.0
        return interp_table_linear(SAC305["E_T"], SAC305["E_GPa"], T) * 1000.0
    Et = grid_table(E)
    Ft = grid_table(lambda T: SAC305["cte"] * (T - T_STRAIN_ORIGIN))
    return Et, Ft


# SAC305 Anand constant set of the stacked-module thermal-cycle workload (s0 = 45.9 MPa, Q/R = 7460 K,
# A = 5.87e6 1/s, xi = 2, m = 0.0942, h0 = 9350 MPa, s_hat = 58.3 MPa, n = 0.015, a = 1.5) with a
# linear E(T) through the database's end points (57.4 GPa at -40 degC, 30.0 GPa at 125 degC)
SAC305_MODULE = dict(A=5.87e6, QR=7460.0, xi=2.0, m=0.0942, shat=58.3, n=0.015, h0=9350.0, a=1.5, s0=45.9, nu=0.4,
                     E_T=[-40.0, 125.0], E_GPa=[57.4, 30.0], solidus=217.0, cte=22.5e-6)


def anand_tables(p: dict):
    """E(T) (MPa, linear table with linear extrapolation, 1 % above the solidus) and F(T) = alpha (T - 25)
    on the 1 degC grid for an Anand parameter set with E_T / E_GPa / solidus / cte entries."""
    def E(T):
        if T > p["solidus"]:
            return 0.01 * interp_table_linear(p["E_T"], p["E_GPa"], p["solidus"]) * 1000.0
        return interp_table_linear(p["E_T"], p["E_GPa"], T) * 1000.0
    return grid_table(E), grid_table(lambda T: p["cte"] * (T - T_STRAIN_ORIGIN))


def anand_params_array(p: dict) -> np.ndarray:
    """Parameter vector (A, Q/R, xi, m, s_hat, n, h0, a, s0, nu) of the Anand entry points."""
    return np.array([p["A"], p["QR"], p["xi"], p["m"], p["shat"], p["n"], p["h0"], p["a"], p["s0"], p["nu"]], np.float64)


def elastic_tables(E_T, E_MPa, cte: float):
    """E(T) (MPa, linear table with linear extrapolation) and F(T) = cte (T - 25) on the 1 degC
    grid, for an elastic material such as a Cu pillar."""
    Et = grid_table(lambda T: interp_table_linear(E_T, E_MPa, T))
    Ft = grid_table(lambda T: cte * (T - T_STRAIN_ORIGIN))
    return Et, Ft



# ---- temperature-dependent properties of a database record -----------------------------------
# (the caller's side in the tool; restated for the host-side known-answer tests and packages)

SIGMOID_W_DEFAULT = 8.0       # 00-constants.js:22
CTE_SMOOTH_DELTA = 3.0        # 00-constants.js:23
PPM = 1e-6
GPA = 1000.0


def _pv(p):
    return p["v"] if isinstance(p, dict) else p


def _mod_mpa(p) -> float:
    """modMPa (03-materials.js:21-25): a modulus parameter in MPa by its unit."""
    u = (p.get("u") if isinstance(p, dict) else None) or "GPa"
    return _pv(p) if u == "MPa" else _pv(p) * GPA


def modulus_at(edef: dict, T: float) -> float:
    """evalEdef (03-materials.js:88-107) for constant and glass-transition (sigmoid) moduli:
    E(T) = E_r + (E_g - E_r) / (1 + exp((T - Tg_DMA) / w))."""
    t = edef["type"]
    if t == "const":
        return _mod_mpa(edef["E"])
    if t == "table":
        scale = 1.0 if edef.get("u") == "MPa" else GPA
        xs, ys = list(edef["T"]), list(edef["v"])
        if (edef.get("extrap") or "hold") != "linear" and len(xs) > 1:
            T = min(max(T, xs[0]), xs[-1])
        if edef.get("interp") == "log":
            return float(np.exp(interp_table_linear(xs, [float(np.log(v)) for v in ys], T))) * scale
        return interp_table_linear(xs, ys, T) * scale
    if t == "sigmoid":
        Eg, Er = _mod_mpa(edef["Eg"]), _mod_mpa(edef["Er"])
        w = _pv(edef.get("w")) or SIGMOID_W_DEFAULT
        return Er + (Eg - Er) / (1 + np.exp((T - _pv(edef["TgDMA"])) / w))
    raise ValueError(f"modulus type {t!r} not restated")


KELVIN = 273.15
CTE_INTEGRATION_SUBSTEPS = 8   # 00-constants.js:14


def iso_modulus(mat: dict, T: float) -> float:
    """isoE (03-materials.js:109-116): the record's E(T), above a solder's solidus 1 % of its
    modulus at the solidus (SOLDER_MOLTEN_FRACTION)."""
    if mat.get("solidus") is not None:
        Ts = _pv(mat["solidus"])
        if T > Ts:
            return 0.01 * modulus_at(mat["elastic"]["E"], Ts)
    return modulus_at(mat["elastic"]["E"], T)


def silicon_alpha(T: float) -> float:
    """Instantaneous CTE of silicon, Okada and Tokumaru (1984) (siliconAlpha, 03-materials.js:132-135)."""
    TK = T + KELVIN
    return (3.725 * (1 - np.exp(-5.88e-3 * (TK - 124))) + 5.548e-4 * TK) * 1e-6


def _simpson(f, a, b, n):
    if n % 2:
        n += 1
    h = (b - a) / n
    s = f(a) + f(b)
    for i in range(1, n):
        s += f(a + i * h) * (4 if i % 2 else 2)
    return s * h / 3


def _softplus(x: float) -> float:
    return x if x > 30 else float(np.log1p(np.exp(x)))


def cte_at(cdef: dict, T: float) -> float:
    """cteAlpha (03-materials.js:138-156), constant, bilinear and tabulated kinds: the bilinear CTE
    switches from a1 to a2 around Tg_TMA by a logistic step of width delta; a table is
    interpolated piecewise linearly (linear extrapolation unless it says 'hold')."""
    t = cdef["type"]
    if t == "const":
        return _pv(cdef["a"]) * PPM
    if t == "silicon":
        return silicon_alpha(T)
    if t == "table":
        xs, ys = cdef["T"], cdef["v"]
        xs = xs["v"] if isinstance(xs, dict) else xs
        ys = ys["v"] if isinstance(ys, dict) else ys
        if (cdef.get("extrap") or "linear") != "linear" and len(xs) > 1:
            T = min(max(T, xs[0]), xs[-1])
        return interp_table_linear(xs, ys, T) * PPM
    if t == "bilinear":
        a1, a2 = _pv(cdef["a1"]) * PPM, _pv(cdef["a2"]) * PPM
        d = _pv(cdef.get("delta")) or CTE_SMOOTH_DELTA
        return a1 + (a2 - a1) / (1 + np.exp(-(T - _pv(cdef["TgTMA"])) / d))
    raise ValueError(f"CTE type {t!r} not restated")


def thermal_strain_at(cdef: dict, T: float) -> float:
    """thermalStrain (03-materials.js:167-195), constant and bilinear kinds: the cumulative
    thermal strain F(T) from 25 degC in closed form (the logistic term integrates to
    (a2 - a1) delta ln(1 + exp((T - Tg) / delta)))."""
    T0 = T_STRAIN_ORIGIN
    t = cdef["type"]
    if t == "const":
        return _pv(cdef["a"]) * PPM * (T - T0)
    if t == "bilinear":
        a1, a2 = _pv(cdef["a1"]) * PPM, _pv(cdef["a2"]) * PPM
        d = _pv(cdef.get("delta")) or CTE_SMOOTH_DELTA
        Tg = _pv(cdef["TgTMA"])
        return a1 * (T - T0) + (a2 - a1) * d * (_softplus((T - Tg) / d) - _softplus((T0 - Tg) / d))
    if t == "table":
        # piecewise-linear alpha: trapezoids between the break points are exact
        lo, hi = min(T, T0), max(T, T0)
        pts = [lo] + [float(x) for x in cdef["T"] if lo < x < hi] + [hi]
        s = 0.0
        for i in range(len(pts) - 1):
            s += 0.5 * (pts[i + 1] - pts[i]) * (cte_at(cdef, pts[i]) + cte_at(cdef, pts[i + 1]))
        return s if T >= T0 else -s
    if t == "silicon":
        n = max(2, 2 * int(np.ceil(abs(T - T0) * CTE_INTEGRATION_SUBSTEPS / 2)))
        return _simpson(silicon_alpha, T0, T, n)
    raise ValueError(f"CTE type {t!r} not restated")


def iso_tables(mat: dict) -> dict:
    """isoTables (03-materials.js:424-433) of an isotropic record: E(T) in MPa and F(T) on the
    1 degC grid, and nu."""
    E = grid_table(lambda T: iso_modulus(mat, T))
    cte = mat.get("cteXY") or mat["cte"]
    F = grid_table(lambda T: thermal_strain_at(cte, T))
    return dict(E=E, F=F, nu=_pv(mat["elastic"]["nu"]))


def material_tgs(mat: dict) -> list:
    """materialTgs (03-materials.js:203-216): the glass transitions of a record (the thermal path
    takes smaller steps around them)."""
    out = []
    el = mat.get("elastic", {})
    if el.get("E", {}).get("type") == "sigmoid":
        out.append(float(_pv(el["E"]["TgDMA"])))
    for c in {id(x): x for x in (mat.get("cteXY") or mat.get("cte"), mat.get("cteZ")) if x}.values():
        if c.get("type") == "bilinear":
            out.append(float(_pv(c["TgTMA"])))
    return out


def for_grid_segments(Ta: float, Tb: float, fn) -> None:
    """forGridSegments (03-materials.js:370-377): the pieces of [Ta, Tb] between 1 degC grid points."""
    lo, hi = min(Ta, Tb), max(Ta, Tb)
    t0 = lo
    while t0 < hi - 1e-12:
        t1 = min(hi, TGRID_MIN + np.floor(t0 - TGRID_MIN + 1e-9) + 1)
        fn(0.5 * (t0 + t1), t0, t1)
        t0 = t1


def grid_mean(arr: np.ndarray, Ta: float, Tb: float) -> float:
    """gridMean (03-materials.js:380-387) of a scalar grid: the mean over the step [Ta, Tb]."""
    L = abs(Tb - Ta)
    if L < 1e-12:
        return grid_at(arr, Ta)
    acc = [0.0]
    for_grid_segments(Ta, Tb, lambda tm, t0, t1: acc.__setitem__(0, acc[0] + (t1 - t0) / L * grid_at(arr, tm)))
    return acc[0]


def grid_modulus_strain_increment(E: np.ndarray, F: np.ndarray, Ta: float, Tb: float) -> float:
    """gridModulusStrainIncrement (03-materials.js:413-418): the integral from Ta to Tb of
    E(T) dF(T), exact for the interpolated tables (midpoint modulus per grid piece)."""
    sg = 1.0 if Tb >= Ta else -1.0
    acc = [0.0]
    for_grid_segments(Ta, Tb, lambda tm, t0, t1: acc.__setitem__(0, acc[0] + grid_at(E, tm) * (grid_at(F, t1) - grid_at(F, t0))))
    return sg * acc[0]


def ortho_factor(el: dict, T: float) -> float:
    """orthoFactor (03-materials.js:119-126): the glass-transition factor on every orthotropic
    modulus, r + (1 - r) / (1 + exp((T - Tg) / w)) with the rubbery ratio r (1 without one)."""
    r, Tg = _pv(el.get("rubberyRatio")), _pv(el.get("TgDMA"))
    if r is None or Tg is None:
        return 1.0
    w = _pv(el.get("w")) or SIGMOID_W_DEFAULT
    return r + (1 - r) / (1 + np.exp((T - Tg) / w))


def material_ec(mat: dict, T: float) -> dict:
    """materialEC (03-materials.js:317-340): engineering constants (MPa, 1/degC) of a database
    record at T, for homogenization: isotropic records with their E(T), orthotropic ones with
    their moduli times the glass-transition factor; in-plane and through-thickness CTEs."""
    el = mat["elastic"]
    cxy = mat.get("cteXY") or mat["cte"]
    cz = mat.get("cteZ") or cxy
    axy, az = cte_at(cxy, T), cte_at(cz, T)
    if el["type"] == "iso":
        ec = iso_ec(modulus_at(el["E"], T), _pv(el["nu"]), axy)
        ec["az"] = az
        return ec
    if el["type"] == "ortho":
        f = ortho_factor(el, T)
        return dict(Ex=f * _mod_mpa(el["Ex"]), Ey=f * _mod_mpa(el["Ey"]), Ez=f * _mod_mpa(el["Ez"]), Gxy=f * _mod_mpa(el["Gxy"]),
                    Gxz=f * _mod_mpa(el["Gxz"]), Gyz=f * _mod_mpa(el["Gyz"]), nuxy=_pv(el["nuxy"]), nuxz=_pv(el["nuxz"]),
                    nuyz=_pv(el["nuyz"]), ax=axy, ay=axy, az=az)
    raise ValueError(f"elastic type {el['type']!r} not restated")
