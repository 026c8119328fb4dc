"""Stacked-module stages in the oracle (assembleStep with moduleStage, moduleStageSet and the
multigrid over the born parts: src/core/09-assembly.js:392-443, 10-solver.js:260-266, 868-876).

Known answer from the reference's own verification of stacked modules (15-verify.js:608-617): on
the first module step the module stands on a statically determinate 3-2-1 support under a
self-equilibrated thermal load, so the support reactions vanish (criterion 1e-6 of the internal
force scale).
"""
import numpy as np

from tmsolve.packages import module_path_steps, stacked_module


def test_module_stage_support_reactions_vanish(oracle_lib):
    pkg = stacked_module(24)
    om = oracle_lib.OracleModel(pkg)
    steps, Tb, chain, up, down = module_path_steps(pkg)
    assert steps[0].stage == -1 and steps[1].stage == 0
    r = om.solve(om.assemble(steps[0]), tol=1e-10, key=0)
    assert r["converged"]
    f = om.assemble(steps[0], no_constraints=True)
    Ku = om.matvec(r["u"])
    mc = pkg.mesh.moduleConstraints
    scale = max(np.abs(Ku).max(), np.abs(f).max())
    assert np.abs(Ku[mc] - f[mc]).max() / scale < 1e-6
    # the package outside the module neither moves nor carries load: every node that no born
    # element touches is held, and those nodes stay out of the multigrid aggregates
    module_elems = pkg.group_stage[pkg.mesh.eGroup] <= -1
    touched = np.zeros(pkg.mesh.nn, bool)
    touched[pkg.mesh.conn.reshape(-1, 8)[module_elems].ravel()] = True
    u = r["u"].reshape(-1, 3)
    assert not u[~touched].any()
    agg = om.mg_node_agg()
    assert np.array_equal(agg >= 0, touched)
    assert om.mg_levels()[1][2] < om.mg_levels()[0][2]


def test_stage_zero_after_module_stage_uses_whole_package(oracle_lib):
    pkg = stacked_module(24)
    om = oracle_lib.OracleModel(pkg)
    steps, *_ = module_path_steps(pkg)
    om.solve(om.assemble(steps[0]), tol=1e-10, key=0)
    lv_mod = om.mg_levels()
    r = om.solve(om.assemble(steps[1]), tol=1e-10, key=1)
    assert r["converged"]
    assert (om.mg_node_agg() >= 0).all()
    assert om.mg_levels()[1][2] > lv_mod[1][2]
