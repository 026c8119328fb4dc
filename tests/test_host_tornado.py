"""Host side of the tornado batch: the case list (sensitivityBounds' relative bounds of matE and
matCTE inputs) and the package's material scaling."""
import numpy as np

from tmsolve.packages import lidded_c2
from tmsolve.sensitivity import SENS_REL, case_scales, tornado_cases


def test_tornado_cases():
    cases = tornado_cases()
    assert len(cases) == 24
    assert [c["factor"] for c in cases[:2]] == [1 - SENS_REL, 1 + SENS_REL]
    assert sum(c["kind"] == "E" for c in cases) == 12 and sum(c["kind"] == "CTE" for c in cases) == 12
    assert case_scales(None) == {}
    assert case_scales(dict(material="cu", kind="CTE", factor=1.1)) == {"cu": (1.0, 1.1)}


def test_material_step_scaling():
    pkg = lidded_c2(n_inplane=8)
    base, same = pkg.step(), pkg.material_step({})
    for k in ("D", "s0", "W", "V"):
        assert np.array_equal(getattr(base, k), getattr(same, k))
    # the die's modulus scales its set's stiffness and thermal stress alike; its CTE only the thermal stress
    die = pkg.npset - 4
    e = pkg.material_step({"die": (1.1, 1.0)})
    a = pkg.material_step({"die": (1.0, 1.1)})
    np.testing.assert_allclose(e.D[36 * die:36 * die + 36], 1.1 * base.D[36 * die:36 * die + 36], rtol=1e-15)
    np.testing.assert_allclose(e.s0[6 * die:6 * die + 6], 1.1 * base.s0[6 * die:6 * die + 6], rtol=1e-14)
    assert np.array_equal(a.D, base.D)
    np.testing.assert_allclose(a.s0[6 * die:6 * die + 6], 1.1 * base.s0[6 * die:6 * die + 6], rtol=1e-14)
    # a substrate material reaches the layered sets only
    c = pkg.material_step({"cu": (1.1, 1.0)})
    assert np.array_equal(c.D, base.D) and not np.array_equal(c.W, base.W)
