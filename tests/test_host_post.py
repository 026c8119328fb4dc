"""Host post-processing readers (tmsolve.post) and their oracle, on the CPU.

* fit_plane, warpage_jeita: the reference's V12 known answer (dome / bowl sign and exact
  magnitude on synthetic surfaces sampled at the balls, 15-verify.js:396-417), an exactly
  recovered plane, and bit-for-bit agreement with the oracle's restatement on a mesh field;
* the oracle's samplePlane + warpageJEITA on a bilinear field (reproduced exactly by the
  interpolation): plane and magnitude to 1e-12 / 1e-9;
* the oracle's strain recovery (accumulateStep qOnly + boxStrainAt): a uniform strain field is
  returned at every natural point and a rigid rotation gives no strain (patch test);
* site generation and the screening subsample rule.
"""
import math

import numpy as np
import pytest

from tmsolve import post
from tmsolve.packages import fcbga_c1


def test_fit_plane_exact_and_oracle(oracle_lib):
    rng = np.random.default_rng(3)
    x = rng.uniform(-10, 10, 200); y = rng.uniform(-10, 10, 200)
    c = post.fit_plane(x, y, 0.25 - 1.5 * x + 0.75 * y)
    assert np.allclose(c, (0.25, -1.5, 0.75), rtol=0, atol=1e-13)
    w = rng.standard_normal(200)
    assert post.fit_plane(x, y, w) == tuple(oracle_lib.fit_plane(x, y, w))
    # degenerate (collinear) points: slopes stay zero, c0 is the mean
    c = post.fit_plane([0, 1, 2], [0, 1, 2], [1.0, 2.0, 3.0])
    assert c == (2.0, 0.0, 0.0)


def test_bump_axis_and_bga_sites():
    assert post.bump_axis(0, 35, 0.75, 1.0) == dict(n=34, first=-16.5, last=16.5)
    assert post.bump_axis(1.0, 0.5, 0.5, 0.2)["n"] == 0
    b = post.bga_sites(35.0, 35.0, 0.75, 1.0)
    assert len(b["x"]) == 34 * 34 and b["zone"] == dict(x0=-16.5, x1=16.5, y0=-16.5, y1=16.5)
    b = post.bga_sites(35.0, 35.0, 0.75, 1.0, depop=dict(on=True, sx=10.0, sy=10.0))
    assert len(b["x"]) == 34 * 34 - 10 * 10
    assert np.all((np.abs(b["x"]) >= 5) | (np.abs(b["y"]) >= 5))


def test_screening_sites_rule():
    d = post.bump_field(0, 0, 25, 25, 0.2, 0.15, 0.15)
    a = post.die_bump_sites(d)
    assert len(a["x"]) == 165 * 165
    r = post.screening_sites(d)
    assert r["subsampled"] and len(r["idx"]) == post.SCREEN_MAX_BUMPS
    assert np.all(np.diff(r["idx"]) > 0)
    cb = post.SCREEN_CORNER_BLOCK
    must = (a["row"] < post.SCREEN_KEEP_ROWS) | (((a["ix"] < cb) | (a["ix"] >= 165 - cb)) & ((a["iy"] < cb) | (a["iy"] >= 165 - cb)))
    assert set(np.nonzero(must)[0]) <= set(r["idx"].tolist())
    small = post.bump_field(0, 0, 15, 15, 0.15, 0.15, 0.15)
    r = post.screening_sites(small)
    assert not r["subsampled"] and len(r["sites"]["x"]) == 99 * 99
    per = post.bump_field(0, 0, 15, 15, 0.15, 0.15, 0.15, rows=4, peripheral=True)
    assert per["peripheral"] and len(post.die_bump_sites(per)["x"]) == 99 * 99 - 91 * 91


@pytest.mark.parametrize("sign", [1, -1])
def test_warpage_v12_dome_bowl(sign):
    """V12: a dome (bowl) sampled exactly at the balls has sign +1 (-1) and magnitude
    c (r2max - r2min) / L^2 to 1e-9."""
    b = post.bga_sites(35.0, 35.0, 0.75, 1.0)
    L, c = 30.0, 0.1
    w = post.warpage_jeita(b, lambda x, y: sign * c * (1 - (x / L) ** 2 - (y / L) ** 2))
    r2 = b["x"] ** 2 + b["y"] ** 2
    an = c * (r2.max() - r2.min()) / (L * L)
    assert w["sign"] == sign and abs(w["mag"] - an) / an < 1e-9
    assert w["shape"] == ("dome" if sign > 0 else "bowl")


def _smooth_field(mesh, seed=5):
    rng = np.random.default_rng(seed)
    X, Y = mesh.coords[0::3], mesh.coords[1::3]
    u = np.zeros(3 * mesh.nn)
    u[2::3] = 0.05 * np.cos(X / 11.0) * np.cos(Y / 13.0) + 1e-3 * X - 2e-3 * Y + 1e-5 * rng.standard_normal(mesh.nn)
    u[0::3] = 1e-4 * rng.standard_normal(mesh.nn); u[1::3] = 1e-4 * rng.standard_normal(mesh.nn)
    return u


def test_warpage_host_matches_oracle(oracle_lib):
    pkg = fcbga_c1()
    om = oracle_lib.OracleModel(pkg)
    b = post.bga_sites(**pkg.meta["bga"])
    u = _smooth_field(pkg.mesh)
    w = post.warpage_jeita(b, lambda x, y: np.array([om.sample_plane(u, 0, 2, a, c) for a, c in zip(x, y)]))
    z = b["zone"]
    o = om.warpage_jeita(u, b["x"], b["y"], [z["x0"], z["x1"], z["y0"], z["y1"]])
    for k in ("signed", "mag", "sign", "signConf", "rmin", "rmax"):
        assert w[k] == o[k], k
    assert tuple(o["plane"]) == w["plane"]


def test_oracle_warpage_bilinear_known_answer(oracle_lib):
    """u_z = a + b x + c y + d x y is reproduced exactly by bilinear interpolation; over the
    symmetric ball grid the fitted plane is (a, b, c) and the magnitude d (max xy - min xy)."""
    pkg = fcbga_c1()
    om = oracle_lib.OracleModel(pkg)
    m = pkg.mesh
    a, bb, c, d = 0.01, 2e-4, -3e-4, 5e-5
    X, Y = m.coords[0::3], m.coords[1::3]
    u = np.zeros(3 * m.nn); u[2::3] = a + bb * X + c * Y + d * X * Y
    b = post.bga_sites(**pkg.meta["bga"])
    z = b["zone"]
    o = om.warpage_jeita(u, b["x"], b["y"], [z["x0"], z["x1"], z["y0"], z["y1"]])
    assert np.allclose(o["plane"], (a, bb, c), rtol=1e-12, atol=1e-15)
    xy = b["x"] * b["y"]
    an = d * (xy.max() - xy.min())
    assert abs(o["mag"] - an) / an < 1e-9
    # a saddle: the two diagonals cancel
    assert o["signConf"] < 1e-6


def _recovery_setup(oracle_lib):
    pkg = fcbga_c1()
    om = oracle_lib.OracleModel(pkg)
    step = pkg.step()
    step.born[:] = 0            # no thermal load on the incompatible modes
    om.assemble(step)
    m = pkg.mesh
    elems = np.nonzero(m.ePart == pkg.meta["bump_layer"]["part"])[0][::37].astype(np.int32)
    return pkg, om, elems


def test_oracle_strain_patch_uniform(oracle_lib):
    pkg, om, elems = _recovery_setup(oracle_lib)
    m = pkg.mesh
    E = np.array([[1e-3, 2e-4, -3e-4], [2e-4, -5e-4, 1e-4], [-3e-4, 1e-4, 7e-4]])   # symmetric strain tensor
    P = m.coords.reshape(-1, 3)
    du = (P @ E.T).reshape(-1)
    q = np.zeros(33 * len(elems))
    om.accumulate_q(du, elems, q)
    q = q.reshape(-1, 33)
    assert np.abs(q[:, 24:]).max() <= 1e-12 * np.abs(q[:, :24]).max()     # no incompatible-mode amplitudes
    nat = np.random.default_rng(2).uniform(-1, 1, (len(elems), 3))
    eps = om.element_strains(elems, q, nat)
    want = np.array([E[0, 0], E[1, 1], E[2, 2], 2 * E[0, 1], 2 * E[1, 2], 2 * E[0, 2]])
    assert np.abs(eps - want).max() <= 1e-12


def test_oracle_strain_patch_rigid(oracle_lib):
    pkg, om, elems = _recovery_setup(oracle_lib)
    P = pkg.mesh.coords.reshape(-1, 3)
    th = 1e-3
    R = np.array([[0, -th, 0.5 * th], [th, 0, -0.2 * th], [-0.5 * th, 0.2 * th, 0]])   # infinitesimal rotation
    du = (P @ R.T + np.array([1e-3, -2e-3, 5e-4])).reshape(-1)
    q = np.zeros(33 * len(elems))
    om.accumulate_q(du, elems, q)
    nat = np.random.default_rng(4).uniform(-1, 1, (len(elems), 3))
    eps = om.element_strains(elems, q.reshape(-1, 33), nat)
    assert np.abs(eps).max() <= 1e-15


def test_site_elements_bump_layer():
    pkg = fcbga_c1()
    m = pkg.mesh
    bl = pkg.meta["bump_layer"]
    d = post.bump_field(**pkg.meta["die"])
    s = post.die_bump_sites(d)
    elem, nat = post.site_elements(m, s["x"], s["y"], bl["zmid"], bl["part"])
    assert np.all(elem >= 0)
    assert np.all(m.ePart[elem] == bl["part"])
    assert np.all(np.abs(nat) <= 1)
    # a site outside the die has no solder element
    e2, _ = post.site_elements(m, [15.0], [15.0], bl["zmid"], bl["part"])
    assert e2[0] == -1
    assert post.find_interval([0.0, 1.0, 2.0], math.nan) == 0


def test_eig_sym3_known_answers():
    assert post.eig_sym3([3.0, 1.0, 2.0, 0, 0, 0]) == (3.0, 2.0, 1.0)
    rng = np.random.default_rng(9)
    for _ in range(20):
        s = rng.standard_normal(6)
        M = np.array([[s[0], s[3], s[5]], [s[3], s[1], s[4]], [s[5], s[4], s[2]]])
        assert np.allclose(post.eig_sym3(s), np.linalg.eigvalsh(M)[::-1], rtol=0, atol=1e-12)


def test_oracle_stress_history_free_expansion(oracle_lib):
    """A homogeneous free body heated uniformly (du = alpha dT x) carries no stress; its strain is
    alpha dT on the diagonal (Model.accumulateStep + stateStress, 09-assembly.js:508-571)."""
    from tmsolve.materials import iso_d
    from tmsolve.packages import box_package, linspace
    a = 20e-6
    pkg = box_package(linspace(0, 2, 4), linspace(0, 1, 3), [0, 0.5, 1.0], [(iso_d(100000.0, 0.3), a, a)],
                      lambda i, j, k: 0, Ta=25.0, Tb=125.0)
    om = oracle_lib.OracleModel(pkg)
    st = pkg.step()
    om.assemble(st); om.set_sublayers(st)
    m = pkg.mesh
    du = (a * 100.0 * m.coords.reshape(-1, 3)).reshape(-1)
    el = np.arange(m.ne, dtype=np.int32)
    stride = post.state_stride(st)
    S = np.zeros(stride * m.ne)
    om.accumulate_state(du, el, stride, S)
    eps, sig = om.state_stress(el, S, stride, np.random.default_rng(1).uniform(-1, 1, (m.ne, 3)))
    assert np.abs(sig).max() <= 1e-12 * 100000.0 * a * 100.0
    assert np.allclose(eps[:, :3], a * 100.0, rtol=1e-12) and np.abs(eps[:, 3:]).max() <= 1e-15


def test_oracle_state_stress_picks_the_sub_layer(oracle_lib):
    """stateStress reads the sub-layer under the natural point (subLayerAt, 09-assembly.js:547-552)."""
    from tmsolve.packages import lidded_c2
    pkg = lidded_c2(n_inplane=8)
    om = oracle_lib.OracleModel(pkg)
    st = pkg.step()
    om.assemble(st); om.set_sublayers(st)
    stride = post.state_stride(st)
    m = pkg.mesh
    p = int(np.argmax(st.sub_n))                 # a layered set with the most sub-layers
    e = int(np.nonzero(pkg.e_pset == p)[0][0])
    k = int(m.eIJK[3 * e + 2])
    off = int(np.sum(st.sub_n[:p])); ns = int(st.sub_n[p])
    S = np.zeros(stride)
    for s in range(ns):
        S[33 + 48 * s + 42:33 + 48 * s + 48] = -(s + 1.0)     # S_th of sub-layer s
    for s in range(ns):
        z0, z1 = st.sub_z[2 * (off + s)], st.sub_z[2 * (off + s) + 1]
        zeta = 2 * (0.5 * (z0 + z1) - m.zs[k]) / (m.zs[k + 1] - m.zs[k]) - 1
        _, sig = om.state_stress([e], S, stride, [[0.1, -0.2, zeta]])
        assert np.all(sig == s + 1.0)
