"""The CPU oracle against the reference's own analytic known-answer tests.

The reference (src/core/15-verify.js) verifies its solve path with closed-form
answers; the published measured values are in its README (README.md:349-366).
These tests pin the oracle to them: the oracle is then the checker of the GPU path.
"""
import json
import math
import os

import numpy as np
import pytest

from tmsolve.materials import SAC305, anand_params_array, iso_d, sac305_tables
from tmsolve.packages import box_package, linspace

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "reference_known_answers.json")


def known():
    with open(GOLDEN) as f:
        return json.load(f)


def centre_curvature(mesh, u, half=5.0):
    """centreCurvature + fitCurvature (15-verify.js:38-46, 12-post.js:133-146)."""
    xs, ys, ws = [], [], []
    for i in range(mesh.nx):
        for j in range(mesh.ny):
            n = mesh.nodeId[(i * mesh.ny + j) * mesh.nz]
            if n < 0 or abs(mesh.xs[i]) > half + 1e-9 or abs(mesh.ys[j]) > half + 1e-9:
                continue
            xs.append(mesh.xs[i]); ys.append(mesh.ys[j]); ws.append(u[3 * n + 2])
    xs, ys, ws = map(np.array, (xs, ys, ws))
    A = np.stack([np.ones_like(xs), xs, ys, xs * xs, ys * ys, xs * ys], 1)
    c = np.linalg.solve(A.T @ A, A.T @ ws)
    return 2 * c[3], 2 * c[4]


def timoshenko():
    """V3's closed form (15-verify.js:175-177)."""
    MA, MB = 130000 / (1 - 0.28), 110000 / (1 - 0.34)
    m, nn, h, da, dT = 1, MA / MB, 1, (2.6 - 16.4) * 1e-6, -100
    return 6 * da * dT * (1 + m) ** 2 / (h * (3 * (1 + m) ** 2 + (1 + m * nn) * (m * m + 1 / (m * nn))))


def v3_package(n=28):
    mats = [(iso_d(110000.0, 0.34), 16.4e-6, 16.4e-6), (iso_d(130000.0, 0.28), 2.6e-6, 2.6e-6)]
    return box_package(linspace(-20, 20, n), linspace(-20, 20, n), [0, 0.25, 0.5, 0.75, 1.0], mats,
                       lambda i, j, k: 0 if k < 2 else 1, Ta=25.0, Tb=-75.0)


def v1_package():
    mats = [(iso_d(130000.0, 0.28), 2.6e-6, 2.6e-6)]
    return box_package(linspace(0, 10, 5), linspace(0, 8, 4), linspace(0, 2, 1), mats, lambda i, j, k: 0, Ta=25.0, Tb=125.0)


def test_v1_free_expansion(oracle_lib):
    pkg = v1_package()
    om = oracle_lib.OracleModel(pkg)
    r = om.solve(om.assemble(pkg.step()), tol=1e-14)
    m = pkg.mesh
    a = 2.6e-6 * 100
    X = m.coords.reshape(-1, 3)
    n0 = m.constraints[0] // 3
    err = np.abs(r["u"].reshape(-1, 3) - a * (X - X[n0])).max() / (a * 10)
    assert err < 1e-9, err  # criterion of 15-verify.js:96 (published 3.3e-12)


def test_v2_patch_test(oracle_lib):
    """Incompatible-mode hex on a distorted 2x2x2 mesh reproduces a linear field (15-verify.js:100-163)."""
    L = oracle_lib.lib()
    D = iso_d(100000.0, 0.3)
    X = np.zeros(27 * 3)
    dist = [0.15, -0.1, 0.12]
    for i in range(3):
        for j in range(3):
            for k in range(3):
                n = (i * 3 + j) * 3 + k
                X[3 * n:3 * n + 3] = [i / 2, j / 2, k / 2]
                if i == 1 and j == 1 and k == 1:
                    X[3 * n:3 * n + 3] += dist
                if i == 1 and j == 1 and k != 1:
                    X[3 * n] += 0.08; X[3 * n + 1] -= 0.05
                if i == 1 and k == 1 and j != 1:
                    X[3 * n] -= 0.06; X[3 * n + 2] += 0.07
                if j == 1 and k == 1 and i != 1:
                    X[3 * n + 1] += 0.09; X[3 * n + 2] -= 0.04
    A = np.array([1e-3, 2e-4, -3e-4, 5e-4, -2e-3, 4e-4, -1e-4, 3e-4, 1.5e-3]).reshape(3, 3)
    exact = lambda n: A @ X[3 * n:3 * n + 3]
    loc = [[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0], [0, 0, 1], [1, 0, 1], [1, 1, 1], [0, 1, 1]]
    K = np.zeros((81, 81))
    recs = []
    for i in range(2):
        for j in range(2):
            for k in range(2):
                nodes = [((i + l[0]) * 3 + j + l[1]) * 3 + k + l[2] for l in loc]
                Xe = np.concatenate([X[3 * n:3 * n + 3] for n in nodes])
                Kc = np.zeros(576); Xc = np.zeros(216)
                L.orc_general_element(Xe, D, Kc, Xc)
                recs.append((nodes, Xe, Xc.reshape(9, 24)))
                Kc = Kc.reshape(24, 24)
                for a in range(8):
                    for b in range(8):
                        K[3 * nodes[a]:3 * nodes[a] + 3, 3 * nodes[b]:3 * nodes[b] + 3] += Kc[3 * a:3 * a + 3, 3 * b:3 * b + 3]
    c = 13
    free = [3 * c, 3 * c + 1, 3 * c + 2]
    rhs = -sum(K[np.ix_(free, range(3 * n, 3 * n + 3))] @ exact(n) for n in range(27) if n != c)
    uc = np.linalg.solve(K[np.ix_(free, free)], rhs)
    scale = np.abs(A).max()
    err = np.abs(uc - exact(c)).max() / scale
    # constant strain in every element at two interior points
    ufull = np.concatenate([uc if n == c else exact(n) for n in range(27)])
    eps_exact = np.array([A[0, 0], A[1, 1], A[2, 2], A[0, 1] + A[1, 0], A[1, 2] + A[2, 1], A[0, 2] + A[2, 0]])
    serr = 0.0
    for nodes, Xe, Xc in recs:
        ue = np.concatenate([ufull[3 * n:3 * n + 3] for n in nodes])
        alpha = -Xc @ ue
        for pt in ([0.3, -0.5, 0.7], [-0.8, 0.2, -0.1]):
            dx = np.zeros(11); dy = np.zeros(11); dz = np.zeros(11)
            L.orc_general_derivs(Xe, pt[0], pt[1], pt[2], dx, dy, dz)
            q = np.concatenate([ue, alpha]).reshape(11, 3)
            e = np.array([dx @ q[:, 0], dy @ q[:, 1], dz @ q[:, 2], dy @ q[:, 0] + dx @ q[:, 1],
                          dz @ q[:, 1] + dy @ q[:, 2], dz @ q[:, 0] + dx @ q[:, 2]])
            serr = max(serr, np.abs(e - eps_exact).max() / scale)
    assert max(err, serr) < 1e-9, (err, serr)  # 15-verify.js:161


def test_v3_bimaterial_curvature(oracle_lib):
    pkg = v3_package()
    om = oracle_lib.OracleModel(pkg)
    r = om.solve(om.assemble(pkg.step()), tol=1e-10)
    assert r["converged"]
    kxx, _ = centre_curvature(pkg.mesh, r["u"])
    kt = timoshenko()
    assert abs(-kxx / kt - 1) < 0.03
    # the reference's published FE curvature (4 significant digits)
    assert f"{-kxx:.4e}" == known()["V3"]["fe_curvature"]


def clt_curvature(layers, dT):
    """Free thermal curvature of a laminate by classical lamination theory (cltCurvature,
    15-verify.js:49-67): plane-stress stiffnesses Q of the layers (bottom to top), their A, B, D
    integrals and thermal resultants, then the 6 x 6 system for mid-plane strains and curvatures."""
    A, B, D = np.zeros((3, 3)), np.zeros((3, 3)), np.zeros((3, 3))
    NT, MT = np.zeros(3), np.zeros(3)
    z0 = -sum(L["t"] for L in layers) / 2
    for L in layers:
        z1 = z0 + L["t"]
        nu21 = L["nu12"] * L["E2"] / L["E1"]
        den = 1 - L["nu12"] * nu21
        Q = np.array([[L["E1"] / den, L["nu12"] * L["E2"] / den, 0], [L["nu12"] * L["E2"] / den, L["E2"] / den, 0], [0, 0, L["G12"]]])
        a = np.array([L["a1"], L["a2"], 0.0])
        h1, h2, h3 = z1 - z0, (z1 ** 2 - z0 ** 2) / 2, (z1 ** 3 - z0 ** 3) / 3
        A += Q * h1; B += Q * h2; D += Q * h3
        s = Q @ a * dT
        NT += s * h1; MT += s * h2
        z0 = z1
    M = np.block([[A, B], [B, D]])
    x = np.linalg.solve(M, np.concatenate([NT, MT]))
    return x[3], x[4]


def v4_package(n=28):
    """V4's asymmetric three-layer laminate (15-verify.js:183-203): an orthotropic layer (Ex 36,
    Ey 20, Ez 12 GPa; Gxy 8, Gxz = Gyz = 5 GPa; nu 0.15 / 0.3 / 0.3; CTE 4 ppm in-plane, 12
    through the thickness) under Cu and Si, two element layers each, cooled by 100 degC."""
    from tmsolve.materials import ortho_d
    O = ortho_d(36000.0, 20000.0, 12000.0, 8000.0, 5000.0, 5000.0, 0.15, 0.3, 0.3, 0.45)
    mats = [(O, 4e-6, 12e-6), (iso_d(110000.0, 0.34), 16.4e-6, 16.4e-6), (iso_d(130000.0, 0.28), 2.6e-6, 2.6e-6)]
    return box_package(linspace(-20, 20, n), linspace(-20, 20, n), [0, 0.15, 0.3, 0.4, 0.5, 0.75, 1.0], mats,
                       lambda i, j, k: 0 if k < 2 else (1 if k < 4 else 2), Ta=25.0, Tb=-75.0)


def test_v4_laminate_vs_clt(oracle_lib):
    pkg = v4_package()
    om = oracle_lib.OracleModel(pkg)
    r = om.solve(om.assemble(pkg.step()), tol=1e-10)
    assert r["converged"]
    kxx, kyy = centre_curvature(pkg.mesh, r["u"])
    kx, ky = clt_curvature([
        dict(t=0.3, E1=36000, E2=20000, nu12=0.15, G12=8000, a1=4e-6, a2=4e-6),
        dict(t=0.2, E1=110000, E2=110000, nu12=0.34, G12=110000 / 2.68, a1=16.4e-6, a2=16.4e-6),
        dict(t=0.5, E1=130000, E2=130000, nu12=0.28, G12=130000 / 2.56, a1=2.6e-6, a2=2.6e-6),
    ], -100)
    ex, ey = abs(-kxx / kx - 1), abs(-kyy / ky - 1)
    assert ex < 0.03 and ey < 0.03
    # the reference's published deviations, at their printed precision
    assert f"{100 * ex:.2f}" == known()["V4"]["kx_err_pct"] and f"{100 * ey:.2f}" == known()["V4"]["ky_err_pct"], (ex, ey)


@pytest.mark.parametrize("case", [0, 1, 2])
def test_v6_anand_saturation(oracle_lib, case):
    T, rate, ref_pub, cf_pub = known()["V6"]["cases"][case]
    Et, _ = sac305_tables()
    P = anand_params_array(SAC305)
    sim = oracle_lib.anand_uniaxial(P, Et, T, rate, 0.05, 400)
    TK = T + 273.15
    z = rate / P[0] * math.exp(P[1] / TK)
    cf = P[4] * z ** P[5] / P[2] * math.asinh(z ** P[3])
    assert abs(sim / cf - 1) < 0.01            # 15-verify.js:245
    assert f"{sim:.2f}" == ref_pub              # published simulated value (README.md:354)
    assert f"{cf:.2f}" == cf_pub                # published closed-form value


def test_anand_series_elastic_limit(oracle_lib):
    """A tiny time step leaves the point elastic: sigma = D_el eps (AnandPoint.step, 13-fatigue.js:67-143)."""
    Et, _ = sac305_tables()
    P = anand_params_array(SAC305)
    state = np.zeros(12); state[6] = SAC305["s0"]
    eps = np.array([1e-5, -2e-5, 3e-5, 1e-5, 0, -1e-5])
    d, sig, D = oracle_lib.anand_step(P, Et, state, eps, 25.0, 1e-12)
    E = Et[25 + 80]; nu = SAC305["nu"]
    Del = iso_d(E, nu, nu_max=0.499).reshape(6, 6)
    assert np.allclose(sig, Del @ eps, rtol=1e-6, atol=1e-9)


def test_series_column_limits(oracle_lib):
    """stepSeriesColumn (13-fatigue.js:178-206) in its two limits: with no pillar (fs = 1) it is
    the free-standing column of stepColumn (to the column Newton tolerance, 1e-3 of the axial
    stress); on a rigid pillar with no thermal strain the cap takes the whole column strain,
    i.e. the column screening of the table with zz, yz, zx divided by fs."""
    from tmsolve.anand import cycle_history, cycling_temps, synthetic_strain_table
    from tmsolve.materials import elastic_tables
    Et, Ft = sac305_tables()
    P = anand_params_array(SAC305)
    hist = cycle_history(-40.0, 125.0, 11.0, 15.0, 3)
    temps = cycling_temps(-40.0, 125.0)
    table, _, _ = synthetic_strain_table(16, temps)
    table = table.ravel()
    dW, dE, _ = oracle_lib.anand_screen(P, Et, Ft, temps, table, hist)
    pE, pF = elastic_tables([-40.0, 125.0], [120000.0, 114000.0], 17e-6)
    W1, E1, _ = oracle_lib.anand_screen_pillar(P, Et, Ft, temps, table, hist, 1.0, 0.34, pE, pF)
    assert np.allclose(W1, dW, rtol=1e-3, atol=0) and np.allclose(E1, dE, rtol=1e-3, atol=0)
    fs = 0.4
    W2, E2, _ = oracle_lib.anand_screen_pillar(P, Et, Ft, temps, table, hist, fs, 0.34, np.full(381, 1e13), np.zeros(381))
    t2 = table.reshape(-1, len(temps), 6).copy()
    t2[:, :, [2, 4, 5]] /= fs
    W3, E3, _ = oracle_lib.anand_screen(P, Et, Ft, temps, t2.ravel(), hist)
    assert np.allclose(W2, W3, rtol=1e-6, atol=0) and np.allclose(E2, E3, rtol=1e-6, atol=0)

