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

from tmsolve.materials import SAC305, anand_params_array, elastic_tables, iso_d, sac305_tables
from tmsolve.submodel import NU_MAX_SUBMODEL, SubmodelSpec, boundary_weights, synthetic_spec

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
