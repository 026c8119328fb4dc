"""Sensitivities on the device: the tornado batch of perturbed materials (the reference's
applySensitivity / runSensitivityCase, src/core/14-sensitivity.js:89-156) and the adjoint gradient of a
bump site's last-cycle dW with respect to the property sets' stiffness and
thermal strain (the peak-bump half of the adjoint sensitivities; the reference's tornado,
src/core/14-sensitivity.js, re-runs a whole analysis per input instead).

The site's dW is a function of its strain table, the table a linear function of the element DOF
history q(T_i) at the cycling sample temperatures, q(T_i) the sum of the DOF increments of the path
steps that reach T_i (the chain, then the branch up to T_i: Analysis.qAlong, 11-analysis.js:298-316),
and every increment a linear function of that step's displacement increment du_k
(Model.accumulateStep, 09-assembly.js:508-533), the solution of K_k du_k = f_k. Backwards:

1. g_i = d dW / d eps(T_i) by forward mode through the screening of the site
   (tm_anand_screen_gradient: every table entry a direction carried through the whole history);
2. d dW / d q(T_i) = B^T g_i (tm_element_strains_adjoint);
3. per step k, h_k = the sum of d dW / d q(T_i) over the temperatures whose history contains k, and
   d dW / d du_k = the transpose of step k's DOF increment applied to h_k (tm_accumulate_q_adjoint);
4. per step k one adjoint solve K_k lambda_k = d dW / d du_k and the per-set sums
   lambda_k^T (f_m - K_m du_k) and lambda_k^T f_m (tm_adjoint_sensitivity), plus the explicit
   dependence of the incompatible modes on the thermal strain of the site element's own set.

The screening's Anand material (constants, E(T) and F(T) tables) is held fixed: the parameters are
the global model's property-set stiffness and thermal-strain scales. The Anand state is carried in
registers through the forward-mode sweep, one direction per thread, so no state is stored.
"""
from __future__ import annotations

import numpy as np

from . import post
from .anand import screen_gradient

SENS_REL = 0.10    # relative perturbation of a sensitivity input (00-constants.js:129)
# the inputs of the C2 tornado: the moduli of six materials, then the expansion coefficients of six
TORNADO_E = ("sr", "diel", "cu", "corecu", "core", "solder")
TORNADO_CTE = ("uf", "die", "tim", "adh", "lid", "cu")


def tornado_cases(e_materials=TORNADO_E, cte_materials=TORNADO_CTE, rel: float = SENS_REL) -> list:
    """The perturbed cases: every listed material's modulus (matE), then every listed material's
    expansion coefficient (matCTE), at the low and the high bound, factors 1 -/+ rel
    (sensitivityBounds, 14-sensitivity.js:113-119)."""
    cases = []
    for kind, names in (("E", e_materials), ("CTE", cte_materials)):
        for nm in names:
            for f in (1.0 - rel, 1.0 + rel):
                cases.append(dict(material=nm, kind=kind, factor=f))
    return cases


def case_scales(case: dict) -> dict:
    """The package's material scales {name: (E factor, CTE factor)} of one case (None: the base)."""
    if case is None:
        return {}
    f = float(case["factor"])
    return {case["material"]: (f, 1.0) if case["kind"] == "E" else (1.0, f)}


def tornado(model, cases, tol: float = 1e-8, precision: str = "mixed", warm: int = 1, key: int = 0,
            Ta=None, Tb=None) -> dict:
    """The base case, then every case of `cases`, in one solve loop on one device model. Each case's
    step is assembled with its materials scaled, gets its own multigrid hierarchy (key + case
    index: a hierarchy kept across a 10 % change of one material needs about twice the
    iterations, which costs more than the set-up) and is solved from the Galerkin projection onto
    the `warm` most recent solutions (the warm start, 10-solver.js:885-926; one stored solution
    costs one operator apply and two dot products, and the previous case is already close). Per
    case: the signed JEITA warpage of the bottom surface over the BGA zone and the RMS warpage of the
    bottom plane, with the solve's record; `swing` lists per input the low and high warpage
    (tornadoFromCases)."""
    pkg = model.pkg
    bga = post.bga_sites(**pkg.meta["bga"])
    from .packages import rms_warpage
    out = []
    for q, case in enumerate([None] + list(cases)):
        st = pkg.material_step(case_scales(case), Ta, Tb)
        r = model.solve(model.assemble_step(st), tol=tol, warm=warm, key=key + q, precision=precision)
        if not r["converged"]:
            raise RuntimeError(f"tornado case {case} did not converge")
        u = r["u"]
        w = post.warpage_jeita(bga, lambda x, y: model.sample_plane(u, 0, 2, x, y))
        out.append(dict(case=case, signed=float(w["signed"]), rms=float(rms_warpage(pkg.mesh, u)), iters=int(r["iters"]),
                        iters0=float(r["iters0"]), warm=int(r["warm"]), rebuilt=bool(r["rebuilt"]), ms=float(r["ms"])))
    base, rest = out[0], out[1:]
    swing = []
    for q in range(0, len(rest) - 1, 2):
        lo, hi = rest[q], rest[q + 1]
        swing.append(dict(material=lo["case"]["material"], kind=lo["case"]["kind"], lo=lo["signed"], hi=hi["signed"],
                          span=abs(hi["signed"] - lo["signed"])))
    return dict(base=base, cases=rest, swing=swing)


def _branch_h(path: post.ThermalPath, gq: dict) -> dict:
    """h_k for every step: the summed derivative with respect to q of every sample temperature whose
    history contains step k (chain steps: all temperatures; a branch step: the temperatures at and
    after it on its branch)."""
    h = {}
    total = sum(gq.values())
    for k in path.chain:
        h[k] = total.copy()
    for br in (path.up, path.down):
        acc = np.zeros(33)
        for k in reversed(br):
            T = float(path.Tb[k])
            if T in gq:
                acc = acc + gq[T]
            h[k] = acc.copy()
    return h


def site_dw_gradient(model, path: post.ThermalPath, u_exact, x: float, y: float, temps, zmid: float, part, params: dict, Etab,
                     Ftab, hist: dict, tol: float = 1e-12, pillar=None) -> dict:
    """dW of the joint at (x, y) (the last cycle of hist) and its derivatives with respect to the
    logarithm of every property set's stiffness (dlogE) and thermal strain (dlogA). path holds the
    steps' data and the increments as the analysis keeps them (float32 values), u_exact the steps'
    FP64 solutions; model is the DeviceModel the path was solved with."""
    mesh = model.pkg.mesh
    elem, nat = post.site_elements(mesh, np.array([x]), np.array([y]), zmid, part)
    e = int(elem[0])
    if e < 0:
        raise ValueError("no element of the joint layer at the site")
    temps = [float(T) for T in temps]
    nt = len(temps)
    qs = post.q_along(model, path, np.array([e], np.int32), temps)
    table = np.array([model.element_strains([e], qs[T], nat)[0] for T in temps])
    g = screen_gradient(params, Etab, Ftab, temps, table, hist, pillar=pillar)
    gq_rows = model.element_strains_adjoint(np.full(nt, e, np.int32), np.repeat(nat, nt, axis=0), g["gW"])
    gq = {T: gq_rows[i] for i, T in enumerate(temps)}
    h = _branch_h(path, gq)
    npset = model.pkg.npset
    dlogE = np.zeros(npset); dlogA = np.zeros(npset)
    pset_e = int(model.pkg.e_pset[e])
    conn = mesh.conn[8 * e:8 * e + 8]
    solves = []
    for k, hk in sorted(h.items()):
        if not np.any(hk):
            continue
        model.assemble_step(path.steps[k])
        gdu, gA = model.accumulate_q_adjoint(np.array([e], np.int32), hk)
        gfull = np.zeros(model.ndof)
        for a in range(8):
            gfull[3 * conn[a]:3 * conn[a] + 3] += gdu[0, 3 * a:3 * a + 3]
        r = model.adjoint_sensitivity(gfull, u_exact[k], tol=tol)
        solves.append(r["adjoint"])
        dlogE += r["dlogE"]
        dlogA += r["dlogA"]
        dlogA[pset_e] += gA[0]
    return dict(dW=g["dW"], dE=g["dE"], dlogE=dlogE, dlogA=dlogA, table=table, gW=g["gW"], elem=e, adjoint_solves=solves)


def scale_step(step, pset: int, stiffness: float = 1.0, thermal: float = 1.0):
    """A copy of a step's property-set data with set pset's stiffness scaled by `stiffness` and its
    thermal strain by `thermal` (homogeneous sets: D and s0; layered sets: W and V)."""
    import copy
    st = copy.deepcopy(step)
    if st.layered[pset]:
        st.W[108 * pset:108 * pset + 108] *= stiffness
        st.V[18 * pset:18 * pset + 18] *= stiffness * thermal
    else:
        st.D[36 * pset:36 * pset + 36] *= stiffness
        st.s0[6 * pset:6 * pset + 6] *= stiffness * thermal
    return st
