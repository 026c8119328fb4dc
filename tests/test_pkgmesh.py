"""The package mesher restated from the reference (``buildPackageMesh``, src/core/06-mesher.js:468-563)
against the reference's published mesh sizes of its default package (lidded single die,
``defaultConfig``, src/core/02-config.js:140-166), README.md:91, :358, :377:

* since element layers go by preset: Draft 65k and Standard 314k DOF, both at their preset h_min;
* before that, four element layers per region at every preset: Draft 77k, Standard 506k DOF;
* Fine: 1.18M DOF, h_min enlarged to 0.138 mm by the 850k cap loop.

The published figures are rounded as printed, so the bars are on the printed digits."""
import numpy as np
import pytest

from tmsolve import pkgmesh as pm
from tmsolve.mesh import PART


@pytest.mark.parametrize("preset, layers, kdof", [("draft", None, 65), ("standard", None, 314), ("draft", 4, 77),
                                                  ("standard", 4, 506)])
def test_published_dof(preset, layers, kdof):
    m, info = pm.build_package_mesh(pm.default_config(), {"preset": preset, "layers": layers})
    assert round(info["nDof"] / 1000) == kdof, info["nDof"]
    assert info["ringRefined"]
    if layers is None:
        # the presets reach their own h_min on the default package (no cap scaling)
        assert not info["scaled"] and info["hmin"] == pm.MESH_PRESETS[preset]["hmin"]


def test_published_fine():
    m, info = pm.build_package_mesh(pm.default_config(), {"preset": "fine"})
    assert round(info["nDof"] / 1e4) == 118, info["nDof"]
    assert info["scaled"] and round(info["hmin"], 3) == 0.138, info["hmin"]


def test_default_geometry():
    """deriveGeometry's z levels and the die's bump field on the default package."""
    g = pm.derive_geometry(pm.default_config(), 2)
    assert abs(g["zt"] - 1.356) < 1e-12                 # 2 x 0.020 + 12 x 0.040 + 2 x 0.018 + 0.8
    assert abs(g["zaf"] - 1.431) < 1e-12
    d = g["dies"][0]
    assert d["nbx"] == 132 and abs(d["field"]["x1"] - 9.9) < 1e-12
    assert abs(g["lid"]["zLidBot"] - (1.431 + 0.775 + 0.05)) < 1e-12 and abs(g["lid"]["footH"] - 0.8) < 1e-12
    assert len(g["sub"]["bands"]) == 6                  # 3 groups x 2 bands


def test_draft_mesh_structure():
    m, info = pm.build_package_mesh(pm.default_config(), {"preset": "draft"})
    assert m.nn * 3 == info["nDof"] and np.all(np.diff(m.colStart) >= 0) and m.colStart[-1] == m.nn
    assert np.all((m.eScale > 0) & (m.eScale <= 1))
    parts = m.ePart
    # solder columns superposed on underfill in the bump layer: two phases in the same cells, scales summing to 1
    c2 = m.cellElems.reshape(-1, 2)
    both = c2[(c2[:, 0] >= 0) & (c2[:, 1] >= 0)]
    assert len(both) > 0
    assert np.all(parts[both[:, 0]] == PART["SOLDER"]) and np.all(parts[both[:, 1]] == PART["UF_BUMP"])
    assert np.allclose(m.eScale[both[:, 0]] + m.eScale[both[:, 1]], 1.0)
    # fillet cells above the active face carry their filled fraction (at least 5 %)
    fil = parts == PART["UF_FILLET"]
    assert fil.any() and m.eScale[fil].min() >= pm.FILLET_FILL_MIN
    # every part of the lidded package is present
    for p in ("SUB", "SOLDER", "UF_BUMP", "UF_FILLET", "DIE", "TIM", "LID", "LIDADH"):
        assert (parts == PART[p]).any(), p
    # the feature lines the multigrid keeps: die edges, lid outer and inner edges on both axes
    assert len(m.featureX) == 6 and len(m.featureY) == 6
    assert sorted(np.round(m.xs[m.featureX], 9)) == [-21.5, -18.5, -10.0, 10.0, 18.5, 21.5]


def test_oracle_solves_reference_draft(oracle_lib):
    """The oracle's MG-PCG on the reference's Draft mesh of its default package (65k DOF, layered
    substrate bands, superposed bump phases, scaled fillet cells, lid foot and plate)."""
    from tmsolve.packages import reference_package
    pkg = reference_package("draft")
    om = oracle_lib.OracleModel(pkg)
    r = om.solve(om.assemble(pkg.step()), tol=1e-10)
    assert r["converged"] and r["relres"] <= 1e-10
    assert r["iters"] < 60, r["iters"]


def test_published_v17_package():
    """V17's small bare-die package (12 x 12 mm substrate, 5 x 5 mm die offset to (0.5, -0.3), Draft
    with a 6k DOF cap, src/core/15-verify.js:536-540): printed as 5.9k DOF under its 6k cap
    (README.md:365), after the cap loop enlarged h_min."""
    cfg = pm.preset_config("bare")
    cfg["substrate"]["sx"] = cfg["substrate"]["sy"] = 12
    cfg["dies"][0].update(sx=5, sy=5, x=0.5, y=-0.3)
    m, info = pm.build_package_mesh(cfg, {"preset": "draft", "cap": 6000})
    assert info["scaled"] and not info["ringRefined"]
    assert info["nDof"] <= 6000 and round(info["nDof"] / 100) == 59, info["nDof"]


@pytest.mark.parametrize("which, variant, parts", [
    ("bare", None, ("SUB", "SOLDER", "UF_BUMP", "UF_FILLET", "DIE")),
    ("stiffener2", None, ("SUB", "SOLDER", "UF_FILLET", "DIE", "STIFF", "STIFFADH")),
    ("offset", None, ("SUB", "DIE", "UF_FILLET")),
    ("coreStudy", "A", ("SUB", "DIE")),
])
def test_preset_packages(which, variant, parts):
    """The reference's presets of monolithic dies mesh at Draft: the parts of each package are there,
    bare packages have no lid, and the two side-by-side dies' 0.2 mm gap (narrower than the fillet
    width) is filled to the fillet height (wedgeHeight's gap rule)."""
    cfg = pm.preset_config(which, variant)
    m, info = pm.build_package_mesh(cfg, {"preset": "draft"})
    for p in parts:
        assert (m.ePart == PART[p]).any(), (which, p)
    if cfg["packageType"] == "bare":
        assert not (m.ePart == PART["LID"]).any() and not info["ringRefined"]
    if which == "stiffener2":
        g = info["geometry"]
        assert len(g["dies"]) == 2
        h, inside = pm.wedge_height(g["dies"], g["uf"]["Wf"], g["uf"]["Hf"], 0.0, 0.0)
        assert inside and abs(h - 0.7 * 0.775) < 1e-12


def test_oracle_solves_reference_draft_homogenized(oracle_lib):
    """The same mesh with the reference's substrate-row homogenization (Cu patterns of their
    residual ratios, core with PTH Cu: orthotropic sub-layers) and anisotropic (100) silicon dies:
    the sections differ from the constant-row ones, and the oracle's MG-PCG converges on them."""
    from tmsolve.packages import reference_package
    pkg0, pkg = reference_package("draft"), reference_package("draft", homogenize=True)
    s0, s1 = pkg0.step(), pkg.step()
    assert s1.W.shape == s0.W.shape and not np.allclose(s1.W, s0.W)
    om = oracle_lib.OracleModel(pkg)
    r = om.solve(om.assemble(s1), tol=1e-10)
    assert r["converged"] and r["iters"] < 60, r["iters"]
