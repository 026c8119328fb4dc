"""Anand screening of solder joints on the GPU (host side).

* ``cycle_history`` restates ``cycleHistory`` (src/core/13-fatigue.js:275-293): ramps in
  steps of at most RAMP_MAX_DT = 5 degC and DWELL_MIN_STEPS = 10 steps per dwell;
  phases are encoded 0 start, 1 ramp up, 2 dwell hot, 3 ramp down, 4 dwell cold.
* ``screen`` is the per-site loop of ``screenJoints`` (13-fatigue.js:395-451) through
  ``tm_anand_screen``.
* ``synthetic_strain_table`` builds a bump-layer strain table with the shape of
  ``siteStrainTable`` (13-fatigue.js:318-347): sites on a die bump grid, strains linear
  in temperature (constant-property thermoelasticity), shear growing with the distance
  to the neutral point.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from ._lib import TmAnandMaterial, TmPillar, check, load

RAMP_MAX_DT = 5        # 00-constants.js:111
DWELL_MIN_STEPS = 10   # 00-constants.js:112
PHASES = {"start": 0, "ramp up": 1, "dwell hot": 2, "ramp down": 3, "dwell cold": 4}


def cycle_history(Tmin: float, Tmax: float, ramp_c_per_min: float, dwell_min: float, cycles: int,
                  ramp_max_dt: float = RAMP_MAX_DT, dwell_steps: int = DWELL_MIN_STEPS) -> dict:
    """cycleHistory (13-fatigue.js:275-293) with its step rules as parameters (the reference's
    RAMP_MAX_DT and DWELL_MIN_STEPS by default; ramp_max_dt = 10, dwell_steps = 3 gives 40 load steps
    per -40/125 degC cycle)."""
    rate = ramp_c_per_min / 60.0
    dwell = dwell_min * 60.0
    t, T, cyc, ph = [0.0], [25.0], [0], [0]
    time = [0.0]

    def ramp(frm, to, c):
        n = max(1, math.ceil(abs(to - frm) / ramp_max_dt))
        dur = abs(to - frm) / rate
        for k in range(1, n + 1):
            time[0] += dur / n
            t.append(time[0]); T.append(frm + (to - frm) * k / n); cyc.append(c)
            ph.append(PHASES["ramp up"] if to > frm else PHASES["ramp down"])

    def hold(Tv, c, label):
        for _ in range(dwell_steps):
            time[0] += dwell / dwell_steps
            t.append(time[0]); T.append(Tv); cyc.append(c); ph.append(PHASES[label])

    for c in range(1, cycles + 1):
        ramp(T[-1], Tmax, c); hold(Tmax, c, "dwell hot")
        ramp(Tmax, Tmin, c); hold(Tmin, c, "dwell cold")
    return dict(t=np.array(t), T=np.array(T), cycle=np.array(cyc, np.int32), phase=np.array(ph, np.int32), cycles=cycles)


def cycling_temps(Tmin: float, Tmax: float, step: float = 10.0) -> np.ndarray:
    """Cycling sample temperatures every CYCLE_DT_STEP (00-constants.js:106) with 25 degC included."""
    ts = set(np.arange(Tmin, Tmax + 1e-9, step).round(9).tolist()) | {Tmin, Tmax, 25.0}
    return np.array(sorted(ts))


def synthetic_strain_table(nsites: int, temps: np.ndarray, seed: int = 20261203, die_half: float = 7.5) -> tuple:
    """(table nsites x ntemps x 6, x, y): strain linear in T about 25 degC per site."""
    rng = np.random.default_rng(seed)
    nb = int(math.ceil(math.sqrt(nsites)))
    g = np.linspace(-die_half, die_half, nb)
    X, Y = np.meshgrid(g, g, indexing="ij")
    x = X.ravel()[:nsites]; y = Y.ravel()[:nsites]
    r = np.hypot(x, y) / (math.sqrt(2) * die_half)
    per_deg = np.zeros((nsites, 6))
    per_deg[:, 0] = 8e-6 * (1 + 0.1 * rng.standard_normal(nsites))
    per_deg[:, 1] = 8e-6 * (1 + 0.1 * rng.standard_normal(nsites))
    per_deg[:, 2] = 26e-6 * (1 + 0.05 * rng.standard_normal(nsites))          # axial (total, incl. thermal)
    per_deg[:, 3] = 1e-6 * rng.standard_normal(nsites)
    per_deg[:, 4] = 3.0e-5 * y / die_half * (0.5 + 0.5 * r)                      # gyz, grows with DNP
    per_deg[:, 5] = 3.0e-5 * x / die_half * (0.5 + 0.5 * r)                      # gzx
    e0 = 1e-4 * rng.standard_normal((nsites, 6))
    table = e0[:, None, :] + per_deg[:, None, :] * (np.asarray(temps)[None, :, None] - 25.0)
    return np.ascontiguousarray(table), x, y


def material(params: dict, Etab: np.ndarray, Ftab: np.ndarray):
    Etab = np.ascontiguousarray(Etab, np.float64); Ftab = np.ascontiguousarray(Ftab, np.float64)
    m = TmAnandMaterial(A=params["A"], QR=params["QR"], xi=params["xi"], m=params["m"], shat=params["shat"], n=params["n"],
                        h0=params["h0"], a=params["a"], s0=params["s0"], nu=params["nu"],
                        Etab=Etab.ctypes.data_as(C.POINTER(C.c_double)), Ftab=Ftab.ctypes.data_as(C.POINTER(C.c_double)))
    return m, (Etab, Ftab)


def screen(params: dict, Etab, Ftab, temps, table, hist) -> tuple:
    """dW, dE, stab per site (screenJoints' per-site loop on the GPU)."""
    m, keep = material(params, Etab, Ftab)
    temps = np.ascontiguousarray(temps, np.float64); table = np.ascontiguousarray(table, np.float64)
    ns = table.size // (6 * len(temps))
    t = np.ascontiguousarray(hist["t"], np.float64); T = np.ascontiguousarray(hist["T"], np.float64)
    cyc = np.ascontiguousarray(hist["cycle"], np.int32); ph = np.ascontiguousarray(hist["phase"], np.int32)
    dW = np.zeros(ns); dE = np.zeros(ns); stab = np.zeros(ns)
    vp = lambda a: a.ctypes.data_as(C.c_void_p)
    check(load().tm_anand_screen(C.byref(m), ns, len(temps), vp(temps), vp(table), len(t), vp(t), vp(T), vp(cyc), vp(ph),
                                 int(hist["cycles"]), vp(dW), vp(dE), vp(stab)))
    return dW, dE, stab


def screen_pillar(params: dict, Etab, Ftab, temps, table, hist, fs: float, pillar_nu: float, pEtab, pFtab) -> tuple:
    """dW, dE, stab per site for joints that are a solder cap (height fraction fs) on an elastic
    pillar (E table pEtab, Poisson ratio pillar_nu, thermal strain table pFtab): screenDdi's
    loop with AnandPoint.stepSeriesColumn (13-fatigue.js:178-206, 369-376), on the GPU."""
    m, keep = material(params, Etab, Ftab)
    pE = np.ascontiguousarray(pEtab, np.float64); pF = np.ascontiguousarray(pFtab, np.float64)
    pil = TmPillar(fs=float(fs), nu=float(pillar_nu), Etab=pE.ctypes.data_as(C.POINTER(C.c_double)),
                   Ftab=pF.ctypes.data_as(C.POINTER(C.c_double)))
    temps = np.ascontiguousarray(temps, np.float64); table = np.ascontiguousarray(table, np.float64)
    ns = table.size // (6 * len(temps))
    t = np.ascontiguousarray(hist["t"], np.float64); T = np.ascontiguousarray(hist["T"], np.float64)
    cyc = np.ascontiguousarray(hist["cycle"], np.int32); ph = np.ascontiguousarray(hist["phase"], np.int32)
    dW = np.zeros(ns); dE = np.zeros(ns); stab = np.zeros(ns)
    vp = lambda a: a.ctypes.data_as(C.c_void_p)
    check(load().tm_anand_screen_pillar(C.byref(m), C.byref(pil), ns, len(temps), vp(temps), vp(table), len(t), vp(t), vp(T),
                                        vp(cyc), vp(ph), int(hist["cycles"]), vp(dW), vp(dE), vp(stab)))
    return dW, dE, stab


def point_step(params: dict, Etab, Ftab, state: np.ndarray, eps: np.ndarray, T: float, dt: float, commit=True):
    """Batched AnandPoint.step (+ commit) of independent points: state (npts, 12) updated in place."""
    m, keep = material(params, Etab, Ftab)
    npts = state.shape[0]
    eps = np.ascontiguousarray(eps, np.float64)
    sig = np.zeros((npts, 6)); D = np.zeros((npts, 36))
    vp = lambda a: a.ctypes.data_as(C.c_void_p)
    check(load().tm_anand_step(C.byref(m), npts, vp(state), vp(eps), float(T), float(dt), vp(sig), vp(D), int(commit)))
    return sig, D


def screen_gradient(params: dict, Etab, Ftab, temps, table_site, hist, pillar=None) -> dict:
    """One site's last-cycle dW and dE and their derivatives with respect to its strain table
    (ntemps x 6) by forward mode on the GPU (tm_anand_screen_gradient). pillar: None, or
    (fs, pillar_nu, pEtab, pFtab) for a solder cap on an elastic pillar."""
    m, keep = material(params, Etab, Ftab)
    temps = np.ascontiguousarray(temps, np.float64)
    tab = np.ascontiguousarray(table_site, np.float64).reshape(-1)
    nt = len(temps)
    if tab.size != 6 * nt:
        raise ValueError("the site table needs 6 strains per temperature")
    t = np.ascontiguousarray(hist["t"], np.float64); T = np.ascontiguousarray(hist["T"], np.float64)
    cyc = np.ascontiguousarray(hist["cycle"], np.int32); ph = np.ascontiguousarray(hist["phase"], np.int32)
    dW = C.c_double(); dE = C.c_double(); gW = np.zeros(6 * nt); gE = np.zeros(6 * nt)
    vp = lambda a: a.ctypes.data_as(C.c_void_p)
    pil = None
    if pillar is not None:
        fs, pnu, pE, pF = pillar
        pE = np.ascontiguousarray(pE, np.float64); pF = np.ascontiguousarray(pF, np.float64)
        keep = keep + (pE, pF)
        pil = TmPillar(fs=float(fs), nu=float(pnu), Etab=pE.ctypes.data_as(C.POINTER(C.c_double)),
                       Ftab=pF.ctypes.data_as(C.POINTER(C.c_double)))
    check(load().tm_anand_screen_gradient(C.byref(m), C.byref(pil) if pil is not None else None, nt, vp(temps), vp(tab), len(t),
                                          vp(t), vp(T), vp(cyc), vp(ph), int(hist["cycles"]), C.byref(dW), C.byref(dE), vp(gW), vp(gE)))
    return dict(dW=dW.value, dE=dE.value, gW=gW.reshape(nt, 6), gE=gE.reshape(nt, 6))
