"""Incremental thermoelastic steps of temperature-dependent materials, host side: the thermal
path the tool steps along and the per-step data of an isotropic material from its 1 degC tables.

* ``thermal_path_points`` restates ``thermalPathPoints`` (src/core/11-analysis.js:50-66): steps of
  at most 30 degC, 10 degC where a step would come within 15 degC of a glass transition, through
  the given stops;
* ``iso_step`` forms what ``FEModel.prepareStep`` (src/core/09-assembly.js:346-365) gives a
  homogeneous group of an isotropic table material: the stiffness averaged over the step
  (``gridMean``) and the thermal stress increment, the integral of D(T) dF(T) over the step
  (``gridStressIncrement``), with D(T) = E(T) D_1(nu);
* ``table_box_package``: a box of one such material (``boxModel``, src/core/15-verify.js:11-17)
  whose steps carry those data.
"""
from __future__ import annotations

from typing import Optional

import numpy as np

from .materials import NU_MAX_GLOBAL, grid_mean, grid_modulus_strain_increment, iso_d, iso_tables
from .packages import Package, StepData, box_package

INC_DT_MAX = 30.0     # 00-constants.js:28
INC_DT_TG = 10.0
INC_TG_BAND = 15.0


def thermal_path_points(Ta: float, Tb: float, tgs, stops=()) -> list:
    """thermalPathPoints (11-analysis.js:50-66)."""
    d = float(np.sign(Tb - Ta))
    pts = [Ta]
    if d == 0:
        return pts
    inner = sorted((T for T in stops if (T - Ta) * d > 1e-9 and (Tb - T) * d > 1e-9), key=lambda T: d * T)
    inner.append(Tb)
    T = Ta
    for S in inner:
        while (S - T) * d > 1e-9:
            lo, hi = min(T, T + d * INC_DT_MAX), max(T, T + d * INC_DT_MAX)
            h = INC_DT_TG if any(tg + INC_TG_BAND > lo and tg - INC_TG_BAND < hi for tg in tgs) else INC_DT_MAX
            nxt = round((T + d * h) * 1e6) / 1e6
            T = nxt if (S - nxt) * d > 1e-9 else S
            pts.append(T)
    return pts


def iso_step(tab: dict, Ta: float, Tb: float):
    """(D 36, s0 6) of an isotropic table material over the step Ta -> Tb."""
    nu = min(tab["nu"], NU_MAX_GLOBAL)
    D1 = iso_d(1.0, nu)
    D = D1 * grid_mean(tab["E"], Ta, Tb)
    eF = grid_modulus_strain_increment(tab["E"], tab["F"], Ta, Tb)
    D1m = D1.reshape(6, 6)
    s0 = (D1m[:, 0] + D1m[:, 1] + D1m[:, 2]) * eF
    return D, s0


def table_box_package(mat: dict, xs, ys, zs, constraints=None, name="table box") -> Package:
    """A box of one isotropic table material (one homogeneous group), steps from its tables."""
    tab = iso_tables(mat)
    pkg = box_package(xs, ys, zs, [(iso_d(1.0, 0.3), 0.0, 0.0)], lambda i, j, k: 0, name=name, constraints=constraints)

    def step_fn(Ta, Tb):
        D, s0 = iso_step(tab, Ta, Tb)
        return StepData(layered=np.zeros(1, np.int32), D=D, s0=s0, W=np.zeros(108), V=np.zeros(18),
                        born=np.ones(1, np.int32), sub_n=np.zeros(1, np.int32), sub_z=np.zeros(0), sub_D=np.zeros(0),
                        sub_s0=np.zeros(0))
    pkg.step_fn = step_fn
    pkg.meta["tables"] = tab
    return pkg
