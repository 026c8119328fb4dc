"""The oracle's bump submodel (BumpSubmodel, 13-fatigue.js:470-1104) pinned by known answers:

* patch test: an elastic cell with the boundary moved by a uniform strain field returns that
  field at every interior node (B-bar hexes reproduce linear fields), to the Newton and inner
  solver tolerances;
* free thermal expansion: boundary = alpha (T - 25) x gives the same field everywhere;
* Anand path: an all-solder cell under a uniform strain history integrates every Gauss point
  like one Anand point driven by that strain (AnandPoint.step, pinned by V6), to the Newton
  tolerance.
"""
import numpy as np
import pytest

from tmsolve.materials import (NU_MAX_GLOBAL, SAC305, TGRID_MIN, anand_params_array, column_d, elastic_tables, iso_d,
                               sac305_tables)
from tmsolve.submodel import NU_MAX_SUBMODEL, SubmodelSpec, boundary_weights, synthetic_spec, uniform_spec

GCONN = [0, 4, 6, 2, 1, 5, 7, 3]


def _uniform_spec(mat, field_fn, ts=(25.0, 125.0), uf_cte=0.0, n=4, nz=5):
    xs = np.linspace(0.0, 0.15, n + 1); ys = np.linspace(-0.1, 0.05, n + 1); zs = np.linspace(1.1, 1.3, nz + 1)
    gxs = np.array([-0.05, 0.2]); gys = np.array([-0.15, 0.1]); gzs = np.array([1.0, 1.4])
    bGlob, bW = boundary_weights(xs, ys, zs, (gxs, gys, gzs, lambda i, j, k: GCONN))
    fields = np.zeros((len(ts), 8, 3))
    for it, T in enumerate(ts):
        for i in range(2):
            for j in range(2):
                for k in range(2):
                    fields[it, (i * 2 + j) * 2 + k] = field_fn(T, np.array([gxs[i], gys[j], gzs[k]]))
    u25 = fields[list(ts).index(25.0)].copy()
    Et, Ft = sac305_tables()
    uf_E, uf_F = elastic_tables([-40.0, 125.0], [8000.0, 8000.0], uf_cte)
    flat = elastic_tables([-40.0, 125.0], [1.0, 1.0], 0.0)[1]
    return SubmodelSpec(xs=xs, ys=ys, zs=zs, cell_mat=np.full(n * n * nz, mat, np.int32), ts=np.array(ts),
                        fields=fields.reshape(-1), u25=u25.reshape(-1), bGlob=bGlob, bW=bW, anand=anand_params_array(SAC305),
                        solder_E=Et, solder_F=Ft, uf_E=uf_E, uf_F=uf_F, uf_nu=0.35,
                        si_D=iso_d(130000.0, 0.28, NU_MAX_SUBMODEL), si_F=flat, sub_D=np.tile(iso_d(25000.0, 0.3, NU_MAX_SUBMODEL), 381),
                        sub_F=np.zeros(3 * 381), zt=1.15, zaf=1.25)


def _node_coords(spec):
    X, Y, Z = np.meshgrid(spec.xs, spec.ys, spec.zs, indexing="ij")
    return np.stack([X.ravel(), Y.ravel(), Z.ravel()], axis=1)


E = np.array([[4e-4, 1e-4, -2e-4], [1e-4, -3e-4, 5e-5], [-2e-4, 5e-5, 6e-4]])


def test_submodel_patch_uniform_strain(oracle_lib):
    spec = _uniform_spec(2, lambda T, x: (T - 25.0) / 100.0 * (E @ x))
    om = oracle_lib.OracleSubmodel(spec)
    ok, newton, dmax = om.step(125.0, 60.0)
    assert ok and dmax == 0
    u = om.u().reshape(-1, 3)
    want = _node_coords(spec) @ E.T
    # to the Newton and inner PCG tolerances (SUB_RES_TOL 1e-6, SUB_INNER_TOL 1e-8)
    assert np.abs(u - want).max() <= 1e-7 * np.abs(want).max()


def test_submodel_free_thermal_expansion(oracle_lib):
    a = 30e-6
    spec = _uniform_spec(2, lambda T, x: a * (T - 25.0) * x, uf_cte=a)
    om = oracle_lib.OracleSubmodel(spec)
    ok, newton, _ = om.step(125.0, 60.0)
    assert ok and newton <= 3            # linear problem: one solve, then the increment test
    u = om.u().reshape(-1, 3)
    want = a * 100.0 * _node_coords(spec)
    assert np.abs(u - want).max() <= 1e-7 * np.abs(want).max()


def test_submodel_solder_points_follow_one_anand_point(oracle_lib):
    Et, Ft = sac305_tables()
    P = anand_params_array(SAC305)
    spec = _uniform_spec(1, lambda T, x: (T - 25.0) / 100.0 * (E @ x), n=2, nz=2)
    om = oracle_lib.OracleSubmodel(spec)
    state = np.zeros(12); state[6] = SAC305["s0"]
    for T in (45.0, 65.0, 85.0):
        ok, _, _ = om.step(T, 120.0)
        assert ok
        f = float(np.interp(T, np.arange(-80, 301), Ft)) - float(np.interp(25.0, np.arange(-80, 301), Ft))
        Et_ = (T - 25.0) / 100.0 * E
        eps = np.array([Et_[0, 0] - f, Et_[1, 1] - f, Et_[2, 2] - f, 2 * Et_[0, 1], 2 * Et_[1, 2], 2 * Et_[0, 2]])
        oracle_lib.anand_step(P, Et, state, eps, T, 120.0)
    W, eb = om.points()
    # the Gauss-point strains carry the Newton tolerance (SUB_RES_TOL 1e-6 on the residual)
    assert np.allclose(W, state[8], rtol=1e-4, atol=0) and np.allclose(eb, state[7], rtol=1e-4, atol=0)
    assert state[8] > 0


def test_submodel_run_small_cell(oracle_lib):
    """A bump cell over one short cycle: plastic work in both interface layers, sub-steps taken."""
    from tmsolve.anand import cycle_history
    spec = synthetic_spec(nxy=4, nz=8)
    om = oracle_lib.OracleSubmodel(spec)
    hist = cycle_history(-40.0, 125.0, 33.0, 5.0, 1)
    r = om.run(hist, 0.8, 0.6)
    assert r["dWdie"] > 0 and r["dWsub"] > 0 and r["steps"] >= len(hist["t"]) - 1
    assert r["dW"] == max(r["dWdie"], r["dWsub"])
    assert np.all(np.isfinite(r["loop"][:, 0]))


# ---- homogenized-layer consistency mode (opts.uniformMaterial, 13-fatigue.js:538, 711-748) ----
# A restatement of the grid integrals for whole-degree step ends (03-materials.js:370-418):
# values at the segment midpoints, by linear interpolation in the 1 degC tables.
def _at(tab, T, stride=1, comp=0):
    x = T - TGRID_MIN
    i = min(int(np.floor(x)), len(tab) // stride - 2)
    t = x - i
    return tab[i * stride + comp] + t * (tab[(i + 1) * stride + comp] - tab[i * stride + comp])


def _segments(Ta, Tb):
    lo, hi = min(Ta, Tb), max(Ta, Tb)
    return [(t0 + 0.5, t0, t0 + 1) for t0 in range(int(lo), int(hi))], (1.0 if Tb >= Ta else -1.0), hi - lo


def _mean(tab, Ta, Tb, n=1):
    seg, _, L = _segments(Ta, Tb)
    return np.array([sum(_at(tab, tm, n, c) for tm, _, _ in seg) / L for c in range(n)])


def _modulus_strain(E, F, Ta, Tb):
    seg, sg, _ = _segments(Ta, Tb)
    return sg * sum(_at(E, tm) * (_at(F, t1) - _at(F, t0)) for tm, t0, t1 in seg)


def _stress_increment(Dtab, Ftab, Ta, Tb):
    seg, sg, _ = _segments(Ta, Tb)
    out = np.zeros(6)
    for tm, t0, t1 in seg:
        D = np.array([_at(Dtab, tm, 36, q) for q in range(36)]).reshape(6, 6)
        dF = np.array([_at(Ftab, t1, 3, c) - _at(Ftab, t0, 3, c) for c in range(3)])
        out += sg * D[:, :3] @ dF
    return out


@pytest.mark.parametrize("Ta, Tb", [(25, 125), (125, 60), (-40, 25)])
def test_submodel_uniform_records(oracle_lib, Ta, Tb):
    """The consistency mode's elastic records against a restatement of _elastic's branches: the
    bump layer as solder columns (columnD) plus underfill (isoD at NU_MAX_GLOBAL) with volume
    fractions fb, 1 - fb; each substrate layer as its sub-layer of the top band, with the band's
    Voigt thickness modulus and Turner-weighted through-thickness thermal strain."""
    spec = uniform_spec(synthetic_spec(nxy=4, nz=8), density=0.3)
    om = oracle_lib.OracleSubmodel(spec)
    assert om.nsolder == 0                      # the solder cells are underfill in this mode
    # bump layer
    fb, nu_s = spec.density, spec.anand[9]
    Es, Eu = _mean(spec.solder_E, Ta, Tb)[0], _mean(spec.uf_E, Ta, Tb)[0]
    Ds, Du = column_d(Es, nu_s), iso_d(Eu, spec.uf_nu, NU_MAX_GLOBAL)
    fs = _modulus_strain(spec.solder_E, spec.solder_F, Ta, Tb) / Es
    fu = _modulus_strain(spec.uf_E, spec.uf_F, Ta, Tb) / Eu
    Dw = fb * Ds + (1 - fb) * Du
    sw = np.array([fb * Ds[6 * r:6 * r + 3].sum() * fs + (1 - fb) * Du[6 * r:6 * r + 3].sum() * fu for r in range(6)])
    D, sth = om.elastic(2, Ta, Tb)
    assert np.allclose(D, Dw, rtol=1e-12, atol=0) and np.allclose(sth, sw, rtol=1e-12, atol=1e-300)
    # substrate layers at heights in each sub-layer
    ns = spec.nsec
    secD = spec.sec_D.reshape(ns, -1); secF = spec.sec_F.reshape(ns, -1)
    Dm = [_mean(secD[q], Ta, Tb, 36) for q in range(ns)]
    Ez = EzF = tt = 0.0
    for q in range(ns):
        tq = spec.sec_z[q][1] - spec.sec_z[q][0]
        fx = _at(secF[q], Tb, 3, 0) - _at(secF[q], Ta, 3, 0)
        fy = _at(secF[q], Tb, 3, 1) - _at(secF[q], Ta, 3, 1)
        sq = _stress_increment(secD[q], secF[q], Ta, Tb)
        Ez += tq * Dm[q][14]; EzF += tq * (sq[2] - Dm[q][12] * fx - Dm[q][13] * fy); tt += tq
    for q in range(ns):
        z = 0.5 * (spec.sec_z[q][0] + spec.sec_z[q][1])
        Dw = Dm[q].copy(); Dw[14] = Ez / tt
        dF = np.array([_at(secF[q], Tb, 3, 0) - _at(secF[q], Ta, 3, 0), _at(secF[q], Tb, 3, 1) - _at(secF[q], Ta, 3, 1),
                       EzF / Ez])
        sw = Dw.reshape(6, 6)[:, :3] @ dF
        D, sth = om.elastic(0, Ta, Tb, z)
        assert np.allclose(D, Dw, rtol=1e-12, atol=1e-300), q
        assert np.allclose(sth, sw, rtol=1e-10, atol=1e-12 * np.abs(sw).max()), q
    # without the mode the bump layer's underfill is the plain isotropic step
    D0, _ = oracle_lib.OracleSubmodel(synthetic_spec(nxy=4, nz=8)).elastic(2, Ta, Tb)
    assert np.allclose(D0, iso_d(Eu, spec.uf_nu, NU_MAX_SUBMODEL), rtol=1e-12, atol=0)


def test_submodel_uniform_cell_steps(oracle_lib):
    """A consistency-mode cell steps like an elastic body: one tangent solve per temperature (the
    increment test then passes), no plastic work, a finite field that follows the boundary."""
    spec = uniform_spec(synthetic_spec(nxy=4, nz=8))
    om = oracle_lib.OracleSubmodel(spec)
    for T in (60.0, 125.0, -40.0):
        ok, newton, dmax = om.step(T, 60.0)
        assert ok and newton <= 3 and dmax == 0
    u = om.u()
    assert np.all(np.isfinite(u)) and np.abs(u).max() > 0


# ---- stress snapshots of the cross-section view (_stressSnapshot, 13-fatigue.js:965-989) ----
def _voigt(Em):
    return np.array([Em[0, 0], Em[1, 1], Em[2, 2], 2 * Em[0, 1], 2 * Em[1, 2], 2 * Em[0, 2]])


def test_snapshot_elastic_patch(oracle_lib):
    """An elastic cell under a uniform strain field: the committed Gauss-point stresses are D eps
    everywhere, and GP_TO_NODE carries a constant field to every node unchanged."""
    spec = _uniform_spec(2, lambda T, x: (T - 25.0) / 100.0 * (E @ x))
    om = oracle_lib.OracleSubmodel(spec)
    ok, _, _ = om.step(125.0, 60.0)
    assert ok
    snap = om.stress_snapshot(125.0)
    assert snap.dtype == np.float32 and snap.shape == (om.ne, 8, 6)
    want = iso_d(8000.0, 0.35, NU_MAX_SUBMODEL).reshape(6, 6) @ _voigt(E)
    assert np.abs(snap - want).max() <= 1e-6 * np.abs(want).max()


def test_snapshot_solder_points(oracle_lib):
    """An all-solder cell under a uniform strain history: every node carries the stress of one
    Anand point driven by that strain, at its committed plastic strain (AnandPoint.stressAt)."""
    Et, Ft = sac305_tables()
    P = anand_params_array(SAC305)
    spec = _uniform_spec(1, lambda T, x: (T - 25.0) / 100.0 * (E @ x), n=2, nz=2)
    om = oracle_lib.OracleSubmodel(spec)
    state = np.zeros(12); state[6] = SAC305["s0"]
    for T in (45.0, 65.0, 85.0):
        ok, _, _ = om.step(T, 120.0)
        assert ok
        f = float(np.interp(T, np.arange(-80, 301), Ft)) - float(np.interp(25.0, np.arange(-80, 301), Ft))
        eps = _voigt((T - 25.0) / 100.0 * E) - np.array([f, f, f, 0, 0, 0])
        _, sig, _ = oracle_lib.anand_step(P, Et, state, eps, T, 120.0)
    snap = om.stress_snapshot(85.0).astype(np.float64)
    # the Gauss-point strains carry the Newton tolerance (SUB_RES_TOL 1e-6 on the residual)
    assert np.abs(snap - sig).max() <= 1e-4 * np.abs(sig).max()


def test_run_snapshots_last_cycle(oracle_lib):
    """run records a snapshot at the end of every ramp and dwell of the last cycle."""
    from tmsolve.anand import cycle_history
    spec = synthetic_spec(nxy=4, nz=8)
    om = oracle_lib.OracleSubmodel(spec)
    hist = cycle_history(-40.0, 125.0, 33.0, 5.0, 2)
    r = om.run(hist, 0.8, 0.6, max_snaps=8)
    ph, cy = np.asarray(hist["phase"]), np.asarray(hist["cycle"])
    n = len(ph)
    ends = [k for k in range(1, n) if cy[k] == 2 and (k == n - 1 or ph[k + 1] != ph[k])]
    assert r["nsnaps"] == len(ends) >= 4
    assert np.array_equal(r["snaps_meta"][:, 0], np.asarray(hist["T"])[ends][:8])
    assert np.array_equal(r["snaps_meta"][:, 3], ph[ends][:8])
    assert np.all(np.isfinite(r["snaps"])) and np.abs(r["snaps"]).max() > 0
