"""Parity of the GPU post-processing entry points (through the C-ABI) with the oracle.

Bars: bit-exact. The sampler, the DOF-history march and the strain evaluation repeat the
reference's operations in the same order without fused multiply-add, so for the same inputs
the GPU returns the oracle's doubles, and the host readers above them (plane fit, JEITA sign,
site strain table) then agree to the last bit as well.
"""
import numpy as np
import pytest

from tmsolve import _lib, post
from tmsolve.packages import fcbga_c1

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def c1(oracle_lib):
    from tmsolve.solver import DeviceModel
    pkg = fcbga_c1()
    return pkg, DeviceModel(pkg), oracle_lib.OracleModel(pkg)


def _field(mesh, seed):
    rng = np.random.default_rng(seed)
    X, Y = mesh.coords[0::3], mesh.coords[1::3]
    u = 1e-4 * rng.standard_normal(3 * mesh.nn)
    u[2::3] += 0.05 * np.cos(X / 11.0) * np.cos(Y / 13.0) + 1e-3 * X
    return u


def test_sample_plane_bit_exact(c1):
    pkg, dm, om = c1
    m = pkg.mesh
    u = _field(m, 1)
    rng = np.random.default_rng(2)
    x = np.concatenate([rng.uniform(-20, 20, 500), m.xs[:5], [np.nan]])
    y = np.concatenate([rng.uniform(-20, 20, 500), m.ys[-5:], [0.0]])
    for k, comp in ((0, 2), (0, 0), (m.nz - 1, 2)):      # the top plane has no nodes outside the die: NaN there
        g = dm.sample_plane(u, k, comp, x, y)
        o = np.array([om.sample_plane(u, k, comp, a, b) for a, b in zip(x, y)])
        assert np.array_equal(np.isnan(g), np.isnan(o))
        assert np.array_equal(g[~np.isnan(g)], o[~np.isnan(o)])
    assert np.isnan(dm.sample_plane(u, m.nz - 1, 2, [16.0], [16.0])[0])
    with pytest.raises(_lib.TmError):
        dm.sample_plane(u, m.nz, 2, x, y)


def test_warpage_gpu_matches_oracle(c1):
    pkg, dm, om = c1
    u = _field(pkg.mesh, 3)
    b = post.bga_sites(**pkg.meta["bga"])
    w = post.warpage_jeita(b, lambda x, y: dm.sample_plane(u, 0, 2, x, y))
    z = b["zone"]
    o = om.warpage_jeita(u, b["x"], b["y"], [z["x0"], z["x1"], z["y0"], z["y1"]])
    for k in ("signed", "mag", "sign", "signConf", "rmin", "rmax"):
        assert w[k] == o[k], k
    assert tuple(o["plane"]) == w["plane"]


def _site_elems(pkg):
    m = pkg.mesh
    bl = pkg.meta["bump_layer"]
    s = post.die_bump_sites(post.bump_field(**pkg.meta["die"]))
    elem, nat = post.site_elements(m, s["x"], s["y"], bl["zmid"], bl["part"])
    return s, elem, nat


def test_accumulate_q_and_strains_bit_exact(c1):
    pkg, dm, om = c1
    _, elem, nat = _site_elems(pkg)
    uniq = np.unique(elem).astype(np.int32)
    rng = np.random.default_rng(7)
    qg = np.zeros(33 * len(uniq)); qo = np.zeros(33 * len(uniq))
    for Ta, Tb in ((150.0, 25.0), (25.0, 125.0)):     # two steps: the DOFs accumulate
        step = pkg.step(Ta, Tb)
        du = rng.standard_normal(dm.ndof).astype(np.float32).astype(np.float64) * 1e-3
        dm.prepare_step(step)
        om.assemble(step)
        dm.accumulate_q(du, uniq, qg)
        om.accumulate_q(du, uniq, qo)
        assert np.array_equal(qg, qo), np.abs(qg - qo).max()
    inv = np.searchsorted(uniq, elem)
    q = qg.reshape(-1, 33)[inv]
    eg = dm.element_strains(elem, q, nat)
    eo = om.element_strains(elem, q, nat)
    assert np.array_equal(eg, eo), np.abs(eg - eo).max()
    # no element at a site: NaN row; an index past the mesh is refused
    qn = np.zeros(66); qo1 = np.zeros(33)
    dm.accumulate_q(np.zeros(dm.ndof), np.array([-1, uniq[0]], np.int32), qn)
    om.accumulate_q(np.zeros(dm.ndof), uniq[:1], qo1)    # du = 0: only the thermal load's modes
    assert np.all(np.isnan(qn[:33])) and np.array_equal(qn[33:], qo1)
    with pytest.raises(_lib.TmError):
        dm.accumulate_q(np.zeros(dm.ndof), np.array([dm.ne], np.int32), np.zeros(33))


def test_site_strain_table_matches_oracle(c1):
    """siteStrainTable over a short thermal path (chain 150 -> 25, up 25 -> 75 -> 125, down
    25 -> -25 -> -55) with the GPU solves' displacement increments kept as float32."""
    pkg, dm, om = c1
    temps = [-55.0, -25.0, 25.0, 75.0, 125.0]
    legs = [(150.0, 25.0), (25.0, 75.0), (75.0, 125.0), (25.0, -25.0), (-25.0, -55.0)]
    steps, du, Tb = [], [], []
    for Ta, Tb_ in legs:
        st = pkg.step(Ta, Tb_)
        f = dm.assemble_step(st)
        r = dm.solve(f, tol=1e-10)
        steps.append(st); du.append(r["u"].astype(np.float32).astype(np.float64)); Tb.append(Tb_)
    path = post.ThermalPath(steps=steps, Tb=Tb, du=du, chain=[0], up=[1, 2], down=[3, 4])
    s, elem, nat = _site_elems(pkg)
    sel = np.arange(0, len(s["x"]), 53)
    sites = dict(x=s["x"][sel], y=s["y"][sel])
    bl = pkg.meta["bump_layer"]
    table = post.site_strain_table(dm, path, sites, temps, bl["zmid"], bl["part"]).reshape(len(sel), len(temps), 6)
    # the oracle, element by element as the reference marches (qAlong per element)
    e_s, nat_s = elem[sel], nat[sel]
    uniq = np.unique(e_s).astype(np.int32)
    base = np.zeros(33 * len(uniq))
    om.assemble(steps[0]); om.accumulate_q(du[0], uniq, base)
    qs = {25.0: base.copy()}
    for br in ([1, 2], [3, 4]):
        st = base.copy()
        for k in br:
            om.assemble(steps[k]); om.accumulate_q(du[k], uniq, st)
            qs[Tb[k]] = st.copy()
    inv = np.searchsorted(uniq, e_s)
    for ti, T in enumerate(temps):
        eo = om.element_strains(e_s, qs[T].reshape(-1, 33)[inv], nat_s)
        assert np.array_equal(table[:, ti, :], eo), (T, np.abs(table[:, ti, :] - eo).max())
    # the strain grows with the temperature distance from 25 degC on both branches
    ezz = np.abs(table[:, :, 2] - table[:, 2:3, 2]).mean(axis=0)
    assert ezz[0] > ezz[1] > 0 and ezz[4] > ezz[3] > 0


def test_accumulate_state_and_stress_bit_exact(oracle_lib):
    """Element stress histories on a layered package (sub-layers of the 8-2-8 substrate bands)
    over two steps, and the stress at points: bit-exact with the oracle."""
    from tmsolve.packages import lidded_c2
    from tmsolve.solver import DeviceModel
    pkg = lidded_c2(n_inplane=24)
    dm, om = DeviceModel(pkg), oracle_lib.OracleModel(pkg)
    m = pkg.mesh
    rng = np.random.default_rng(11)
    elems = np.unique(rng.integers(0, m.ne, 400)).astype(np.int32)
    st0 = pkg.step()
    stride = post.state_stride(st0)
    Sg = np.zeros(stride * len(elems)); So = np.zeros(stride * len(elems))
    for Ta, Tb in ((150.0, 25.0), (25.0, 125.0)):
        st = pkg.step(Ta, Tb)
        du = rng.standard_normal(dm.ndof).astype(np.float32).astype(np.float64) * 1e-3
        dm.prepare_step(st); dm.set_sublayers(st)
        om.assemble(st); om.set_sublayers(st)
        dm.accumulate_state(du, elems, stride, Sg)
        om.accumulate_state(du, elems, stride, So)
        assert np.array_equal(Sg, So), np.abs(Sg - So).max()
    nat = rng.uniform(-1, 1, (len(elems), 3))
    eg, sg = dm.state_stress(elems, Sg, stride, nat)
    eo, so = om.state_stress(elems, So, stride, nat)
    assert np.array_equal(eg, eo) and np.array_equal(sg, so)
    assert np.abs(sg).max() > 0
    with pytest.raises(_lib.TmError):
        dm.accumulate_state(du, elems, 33, np.zeros(33 * len(elems)))     # stride below the sub-layers


def test_joint_loads_and_die_stress_match_oracle(c1, oracle_lib):
    """jointLoads and dieSurfaceStress (12-post.js:178-299) from the element histories of a short
    thermal path: the host readers driven by the GPU states equal those driven by the oracle's."""
    pkg, dm, om = c1
    legs = [(150.0, 25.0), (25.0, 125.0)]
    steps, du, Tb = [], [], []
    for Ta, Tb_ in legs:
        st = pkg.step(Ta, Tb_)
        r = dm.solve(dm.assemble_step(st), tol=1e-10)
        steps.append(st); du.append(r["u"].astype(np.float32).astype(np.float64)); Tb.append(Tb_)
    path = post.ThermalPath(steps=steps, Tb=Tb, du=du, chain=[0], up=[1])
    m = pkg.mesh
    stride = post.state_stride(steps[0])
    # the elements the readers visit: bump-layer solder and the die's top and bottom layers
    s, elem, nat = _site_elems(pkg)
    rect = dict(x0=-7.5, x1=7.5, y0=-7.5, y1=7.5)
    zb, ztop = 1.28, float(m.zs[-1])
    die_top, _ = post.die_elements(m, rect, post.plane_index(m, ztop) - 1, 4, 3)
    die_bot, _ = post.die_elements(m, rect, post.plane_index(m, zb), 4, 3)
    uniq = np.unique(np.concatenate([elem[elem >= 0], [e for _, _, e in die_top], [e for _, _, e in die_bot]])).astype(np.int32)
    states = post.states_along(dm, path, uniq, [25.0, 125.0], stride)
    base = np.zeros(stride * len(uniq))
    om.assemble(steps[0]); om.set_sublayers(steps[0]); om.accumulate_state(du[0], uniq, stride, base)
    o125 = base.copy()
    om.assemble(steps[1]); om.set_sublayers(steps[1]); om.accumulate_state(du[1], uniq, stride, o125)
    assert np.array_equal(states[25.0].reshape(-1), base) and np.array_equal(states[125.0].reshape(-1), o125)
    bl = pkg.meta["bump_layer"]
    A = 0.25 * np.pi * 0.09 ** 2
    sites = dict(x=s["x"][::7], y=s["y"][::7])
    jg = post.joint_loads(dm, states[125.0], uniq, stride, sites, bl["zmid"], bl["part"], A)
    jo = post.joint_loads(om, o125.reshape(len(uniq), stride), uniq, stride, sites, bl["zmid"], bl["part"], A)
    assert np.array_equal(jg["N"], jo["N"]) and np.array_equal(jg["V"], jo["V"]) and jg["worst"] == jo["worst"]
    assert np.all(np.isfinite(jg["N"]))
    for which in ("top", "bottom"):
        dg = post.die_surface_stress(dm, states[125.0], uniq, stride, rect, ztop, zb, 4, 3, which)
        do = post.die_surface_stress(om, o125.reshape(len(uniq), stride), uniq, stride, rect, ztop, zb, 4, 3, which)
        assert np.array_equal(dg["smax"], do["smax"], equal_nan=True)
        assert dg["peakInterior"] == do["peakInterior"] and dg["corners"] == do["corners"] and dg["midEdges"] == do["midEdges"]
        assert np.isfinite(dg["peakInterior"])
