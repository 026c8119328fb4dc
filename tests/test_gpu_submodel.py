"""The bump submodel on the GPU (tm_submodel_*) against the oracle's BumpSubmodel.

Bars: one Newton step's tangent and residual repeat the reference's sums, but the inner
IC(0)-PCG sums its dots in another order, so the converged states agree to the solver
tolerances: displacements to 1e-7 and Gauss-point W to 1e-6 relative after single steps; the
cycle run's dW, dWdie, dWsub and dE to 1e-6 relative (the submodel bar), with the same sub-step
and cutback decisions.
"""
import numpy as np
import pytest

from tmsolve.anand import cycle_history
from tmsolve.submodel import DeviceSubmodel, synthetic_spec, uniform_spec

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def test_submodel_patch_and_expansion_gpu(oracle_lib):
    import test_oracle_submodel as T
    spec = T._uniform_spec(2, lambda t, x: (t - 25.0) / 100.0 * (T.E @ x))
    dm = DeviceSubmodel(spec)
    ok, newton, dmax = dm.step(125.0, 60.0)
    assert ok and dmax == 0
    want = T._node_coords(spec) @ T.E.T
    assert np.abs(dm.u().reshape(-1, 3) - want).max() <= 1e-7 * np.abs(want).max()
    a = 30e-6
    spec = T._uniform_spec(2, lambda t, x: a * (t - 25.0) * x, uf_cte=a)
    dm = DeviceSubmodel(spec)
    ok, _, _ = dm.step(125.0, 60.0)
    want = a * 100.0 * T._node_coords(spec)
    assert ok and np.abs(dm.u().reshape(-1, 3) - want).max() <= 1e-7 * np.abs(want).max()


def test_submodel_steps_match_oracle(oracle_lib):
    spec = synthetic_spec(nxy=6, nz=8)
    dm, om = DeviceSubmodel(spec), oracle_lib.OracleSubmodel(spec)
    assert (dm.nn, dm.ne, dm.nb, dm.npoints) == (om.nn, om.ne, om.nb, om.nsolder)
    for T in (30.0, 35.0, 40.0, 30.0):
        g, o = dm.step(T, 30.0), om.step(T, 30.0)
        assert g[0] and o[0]
        assert abs(g[1] - o[1]) <= 1
        assert abs(g[2] - o[2]) <= 1e-6 * o[2]
        assert _rel(dm.u(), om.u()) <= 1e-7
        Wg, Eg = dm.points(); Wo, Eo = om.points()
        assert _rel(Wg, Wo) <= 1e-6 and _rel(Eg, Eo) <= 1e-6


def test_submodel_run_matches_oracle(oracle_lib):
    spec = synthetic_spec(nxy=4, nz=8)
    hist = cycle_history(-40.0, 125.0, 33.0, 5.0, 1)
    rg = DeviceSubmodel(spec).run(hist, 0.8, 0.6)
    ro = oracle_lib.OracleSubmodel(spec).run(hist, 0.8, 0.6)
    for k in ("dW", "dWdie", "dWsub", "dE", "dEdie", "dEsub"):
        assert abs(rg[k] - ro[k]) <= 1e-6 * abs(ro[k]), (k, rg[k], ro[k])
    assert rg["steps"] == ro["steps"] and rg["cutbacks"] == ro["cutbacks"]
    assert np.allclose(rg["loop"], ro["loop"], rtol=1e-5, atol=1e-9)


def _batch_specs():
    # cells of different sizes, so the batched launches map CTAs to uneven submodels
    return [synthetic_spec(nxy=4 + 2 * (q % 2), nz=6 + q, site=(0.3 * q, -0.2 * q), shear=1e-5 * (q + 1), seed=q) for q in range(3)]


@pytest.mark.parametrize("precond", ["ic", "line"])
def test_submodel_batch_equals_single_runs(precond):
    """Three sites of different cell sizes in one batch (every Newton phase one launch over all
    three) give each site's single-run record bit for bit, with either preconditioner."""
    from tmsolve.submodel import run_batch
    hist = cycle_history(-40.0, 125.0, 66.0, 2.0, 1)
    specs = _batch_specs()
    cph, sph = [1.0, 0.6, 0.0], [0.0, 0.8, 1.0]
    models = [DeviceSubmodel(s) for s in specs]
    for m in models:
        m.set_precond(precond)
    recs = run_batch(models, hist, cph, sph)
    for q in range(3):
        one = DeviceSubmodel(specs[q])
        one.set_precond(precond)
        r1 = one.run(hist, cph[q], sph[q])
        for k in ("dW", "dWdie", "dWsub", "dE", "steps", "cutbacks", "newtonPerStep"):
            assert recs[q][k] == r1[k], (q, k)
        assert np.array_equal(recs[q]["loop"], r1["loop"])
        assert np.array_equal(models[q].u(), one.u())


def test_submodel_line_preconditioner_matches_oracle(oracle_lib):
    """The z-line block-Jacobi inner solves against the oracle's IC(0) ones: the inner solves stop
    at the same relative residual, so the Newton iterates agree to the solver tolerances; the run's
    dW, dWdie, dWsub and dE within 1e-6 relative (the submodel bar) with the same sub-steps."""
    spec = synthetic_spec(nxy=4, nz=8)
    hist = cycle_history(-40.0, 125.0, 33.0, 5.0, 1)
    dm = DeviceSubmodel(spec)
    dm.set_precond("line")
    rg = dm.run(hist, 0.8, 0.6)
    ro = oracle_lib.OracleSubmodel(spec).run(hist, 0.8, 0.6)
    for k in ("dW", "dWdie", "dWsub", "dE", "dEdie", "dEsub"):
        assert abs(rg[k] - ro[k]) <= 1e-6 * abs(ro[k]), (k, rg[k], ro[k])
    assert rg["steps"] == ro["steps"] and rg["cutbacks"] == ro["cutbacks"]



def test_submodel_uniform_matches_oracle(oracle_lib):
    """The homogenized-layer consistency mode (opts.uniformMaterial, the V7 check) on the GPU:
    solder cells as the homogenized bump layer, substrate layers from the top band's section."""
    spec = uniform_spec(synthetic_spec(nxy=6, nz=8))
    dm, om = DeviceSubmodel(spec), oracle_lib.OracleSubmodel(spec)
    assert dm.npoints == 0 and om.nsolder == 0
    for T in (60.0, 125.0, -40.0):
        g, o = dm.step(T, 60.0), om.step(T, 60.0)
        assert g[0] and o[0] and abs(g[1] - o[1]) <= 1 and g[2] == 0
        assert _rel(dm.u(), om.u()) <= 1e-7


def test_stress_snapshots_match_oracle(oracle_lib):
    """The section record's stress snapshots (_stressSnapshot): after single steps, and the ones
    run takes at the end of every ramp and dwell of the last cycle. The states agree to the
    solver tolerances, so the float32 nodal stresses do too (1e-6 of the largest after steps,
    1e-5 after a run)."""
    spec = synthetic_spec(nxy=6, nz=8)
    dm, om = DeviceSubmodel(spec), oracle_lib.OracleSubmodel(spec)
    for T in (30.0, 35.0, 40.0):
        assert dm.step(T, 30.0)[0] and om.step(T, 30.0)[0]
        g, o = dm.stress_snapshot(T), om.stress_snapshot(T)
        assert g.shape == o.shape == (om.ne, 8, 6)
        assert _rel(g.astype(np.float64), o.astype(np.float64)) <= 1e-6
    spec = synthetic_spec(nxy=4, nz=8)
    hist = cycle_history(-40.0, 125.0, 33.0, 5.0, 1)
    rg = DeviceSubmodel(spec).run(hist, 0.8, 0.6, max_snaps=8)
    ro = oracle_lib.OracleSubmodel(spec).run(hist, 0.8, 0.6, max_snaps=8)
    assert rg["nsnaps"] == ro["nsnaps"] >= 4
    assert np.array_equal(rg["snaps_meta"], ro["snaps_meta"])
    assert _rel(rg["snaps"].astype(np.float64), ro["snaps"].astype(np.float64)) <= 1e-5
