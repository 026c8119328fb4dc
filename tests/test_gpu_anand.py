"""Anand screening on the GPU against the oracle's restatement of screenJoints' per-site
loop (13-fatigue.js:395-451). Bar: per-site dW and dE within 1e-8 relative (same time
history, FP64 on both sides)."""
import numpy as np
import pytest

from tmsolve.anand import cycle_history, cycling_temps, point_step, screen, screen_pillar, synthetic_strain_table
from tmsolve.materials import SAC305, anand_params_array, elastic_tables, sac305_tables

pytestmark = pytest.mark.gpu


def test_screen_parity(oracle_lib):
    Et, Ft = sac305_tables()
    hist = cycle_history(-40.0, 125.0, 11.0, 15.0, 3)
    temps = cycling_temps(-40.0, 125.0)
    table, x, y = synthetic_strain_table(96, temps)
    table = table.ravel()
    table[6 * len(temps) * 5] = np.nan     # a site outside the bump layer is skipped
    dW, dE, stab = screen(SAC305, Et, Ft, temps, table, hist)
    oW, oE, ostab = oracle_lib.anand_screen(anand_params_array(SAC305), Et, Ft, temps, table, hist)
    assert np.isnan(dW[5]) and np.isnan(oW[5])
    ok = np.isfinite(oW)
    assert np.all(oW[ok] > 0)
    assert np.allclose(dW[ok], oW[ok], rtol=1e-8, atol=0)
    assert np.allclose(dE[ok], oE[ok], rtol=1e-8, atol=0)


def test_screen_pillar_parity(oracle_lib):
    """DDI joints: solder caps (fs = 0.4) on Cu pillars (stepSeriesColumn)."""
    Et, Ft = sac305_tables()
    pE, pF = elastic_tables([-40.0, 125.0], [120000.0, 114000.0], 17e-6)
    hist = cycle_history(-40.0, 125.0, 11.0, 15.0, 3)
    temps = cycling_temps(-40.0, 125.0)
    table, x, y = synthetic_strain_table(64, temps, seed=11)
    table = table.ravel()
    table[6 * len(temps) * 3] = np.nan
    dW, dE, stab = screen_pillar(SAC305, Et, Ft, temps, table, hist, 0.4, 0.34, pE, pF)
    oW, oE, ostab = oracle_lib.anand_screen_pillar(anand_params_array(SAC305), Et, Ft, temps, table, hist, 0.4, 0.34, pE, pF)
    assert np.isnan(dW[3]) and np.isnan(oW[3])
    ok = np.isfinite(oW)
    assert np.all(oW[ok] > 0)
    assert np.allclose(dW[ok], oW[ok], rtol=1e-8, atol=0)
    assert np.allclose(dE[ok], oE[ok], rtol=1e-8, atol=0)
    with pytest.raises(Exception):
        screen_pillar(SAC305, Et, Ft, temps, table, hist, 0.0, 0.34, pE, pF)


def test_point_step_parity(oracle_lib):
    Et, Ft = sac305_tables()
    P = anand_params_array(SAC305)
    rng = np.random.default_rng(3)
    npts = 32
    eps = 2e-3 * rng.standard_normal((npts, 6))
    state = np.zeros((npts, 12)); state[:, 6] = SAC305["s0"]
    sig, D = point_step(SAC305, Et, Ft, state, eps, 75.0, 30.0)
    for q in range(npts):
        st = np.zeros(12); st[6] = SAC305["s0"]
        d, so, Do = oracle_lib.anand_step(P, Et, st, eps[q], 75.0, 30.0)
        assert np.allclose(sig[q], so, rtol=1e-9, atol=1e-9)
        assert np.allclose(state[q, :11], st[:11], rtol=1e-9, atol=1e-12)
        # the consistent tangent (_dsdd, 13-fatigue.js:209-218) that the submodel's Newton uses:
        # within 1e-8 of its largest entry
        assert np.allclose(D[q], Do, rtol=0, atol=1e-8 * np.abs(Do).max()), np.abs(D[q] - Do).max()
    assert np.any(state[:, 7] > 0)      # some points flowed plastically (the tangent is not the elastic one)
