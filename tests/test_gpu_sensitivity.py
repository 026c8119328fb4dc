"""Adjoint warpage sensitivities (tm_warpage_sensitivity) against central finite differences of
full re-solves, on a homogeneous package and a layered one.

Bar: relative 1e-4 against central differences with a relative step of 1e-3 (solves to relative
residual 1e-12; the step's truncation error is ~1e-6 relative, and a smaller step lets the solves'
rounding dominate the difference), for every sensitivity above 1e-3 of the largest of its kind.
"""
import numpy as np
import pytest

from tmsolve.packages import fcbga_c1, lidded_c2

pytestmark = pytest.mark.gpu


def warpage_measure(mesh, u, k=0):
    """Mean squared residual of plane k's z displacements about their least-squares plane."""
    ids = mesh.nodeId.reshape(mesh.nx, mesh.ny, mesh.nz)[:, :, k]
    X, Y = np.meshgrid(mesh.xs, mesh.ys, indexing="ij")
    on = ids >= 0
    w = u[3 * ids[on] + 2]
    A = np.stack([np.ones(on.sum()), X[on], Y[on]], axis=1)
    c = np.linalg.lstsq(A, w, rcond=None)[0]
    r = w - A @ c
    return float(np.mean(r * r))


def _scaled(step, p, kind, f):
    s = type(step)(**{k: (v.copy() if isinstance(v, np.ndarray) else v) for k, v in step.__dict__.items()})
    if s.layered[p]:
        if kind == "E":
            s.W[108 * p:108 * p + 108] *= f
        s.V[18 * p:18 * p + 18] *= f
    else:
        if kind == "E":
            s.D[36 * p:36 * p + 36] *= f
        s.s0[6 * p:6 * p + 6] *= f
    return s


@pytest.mark.parametrize("make", [fcbga_c1, lambda: lidded_c2(n_inplane=24)], ids=["c1", "c2_24"])
def test_adjoint_matches_central_differences(make):
    from tmsolve.solver import DeviceModel
    pkg = make()
    dm = DeviceModel(pkg)
    step = pkg.step()
    r = dm.solve(dm.assemble_step(step), tol=1e-12, warm=0, key=0)
    s = dm.warpage_sensitivity(r["u"], 0, tol=1e-12)
    assert s["adjoint"]["converged"]
    assert abs(s["J"] / warpage_measure(pkg.mesh, r["u"]) - 1) < 1e-9
    h = 1e-3
    key = 1
    for kind, g in (("E", s["dlogE"]), ("A", s["dlogA"])):
        big = np.abs(g).max()
        for p in range(pkg.npset):
            if abs(g[p]) < 1e-3 * big:
                continue
            Js = []
            for f in (1 + h, 1 - h):
                rr = dm.solve(dm.assemble_step(_scaled(step, p, kind, f)), tol=1e-12, warm=0, key=key)
                key += 1
                Js.append(warpage_measure(pkg.mesh, rr["u"]))
            fd = (Js[0] - Js[1]) / (np.log(1 + h) - np.log(1 - h))
            assert abs(g[p] - fd) <= 1e-4 * abs(fd), (kind, p, g[p], fd)


def test_direction_sensitivities_stiffness_and_poisson():
    """tm_sensitivity_direction: along the sets' own data it reproduces dJ/dlog(E); along dD/dnu
    (isotropic and column stiffnesses of the homogeneous package) it matches central differences
    of re-solves in nu."""
    from tmsolve.materials import column_d, iso_d, thermal_stress_const
    from tmsolve.packages import StepData
    from tmsolve.solver import DeviceModel
    pkg = fcbga_c1()
    dm = DeviceModel(pkg)
    step = pkg.step()
    r = dm.solve(dm.assemble_step(step), tol=1e-12, warm=0, key=0)
    s = dm.warpage_sensitivity(r["u"], 0, tol=1e-12)
    same = dm.sensitivity_direction(step, step)
    assert np.allclose(same, s["dlogE"], rtol=1e-6, atol=1e-9 * np.abs(s["dlogE"]).max())
    # the package's sets: (kind, E, nu, alpha) as fcbga_c1 builds them
    mats = [("iso", 25000.0, 0.3, 15e-6), ("col", 40000.0, 0.4, 22.5e-6), ("iso", 8000.0, 0.35, 30e-6), ("iso", 130000.0, 0.28, 2.6e-6)]
    Dof = lambda kind, E, nu: iso_d(E, nu) if kind == "iso" else column_d(E, nu)
    Ta, Tb = pkg.Ta, pkg.Tb

    def step_with(nus):
        D = np.concatenate([Dof(k, E, nu) for (k, E, _, _), nu in zip(mats, nus)])
        s0 = np.concatenate([thermal_stress_const(Dof(k, E, nu), a, a, Ta, Tb) for (k, E, _, a), nu in zip(mats, nus)])
        return StepData(layered=step.layered, D=D, s0=s0, W=step.W, V=step.V, born=step.born, stage=step.stage)
    nus = [m[2] for m in mats]
    d = 1e-7
    dD = [(Dof(k, E, nu + d) - Dof(k, E, nu - d)) / (2 * d) for (k, E, nu, _) in mats]
    direction = StepData(layered=step.layered, D=np.concatenate(dD),
                         s0=np.concatenate([thermal_stress_const(x, a, a, Ta, Tb) for x, (_, _, _, a) in zip(dD, mats)]),
                         W=np.zeros_like(step.W), V=np.zeros_like(step.V), born=step.born, stage=step.stage)
    base = step_with(nus)
    assert np.allclose(base.D, step.D, rtol=1e-14, atol=0)
    r = dm.solve(dm.assemble_step(base), tol=1e-12, warm=0, key=1)
    dm.warpage_sensitivity(r["u"], 0, tol=1e-12)
    g = dm.sensitivity_direction(base, direction)
    h = 1e-3
    key = 2
    for p in range(len(mats)):
        if abs(g[p]) < 1e-3 * np.abs(g).max():
            continue
        Js = []
        for sg in (1, -1):
            nn = list(nus); nn[p] += sg * h
            rr = dm.solve(dm.assemble_step(step_with(nn)), tol=1e-12, warm=0, key=key)
            key += 1
            Js.append(warpage_measure(pkg.mesh, rr["u"]))
        fd = (Js[0] - Js[1]) / (2 * h)
        assert abs(g[p] - fd) <= 1e-4 * abs(fd), (p, g[p], fd)
