"""The tool's process chain on its default package, on the host and the oracle, against the
reference's published whole-package result: the as-assembled warpage at room temperature of
the default lidded single die at the Draft preset, -69.34 um (README.md:91, the per-preset layers
of PR 40; the JEITA signed warpage at 25 degC after the chain 217 -> 165 degC (S1: die and
solder), 165 -> 150 (S2: underfill), 150 -> 25 (S3: lid, TIM, adhesive)).

Everything on the path is the restated model-building side: the mesh (``pkgmesh``), the
substrate bands and the parts' tables from the database records of the default package's
materials (tests/golden/materials_subset.json, extracted by make_material_fixtures.py), the
thermal path with its births, solved step by step by the oracle."""
import json
import os

import numpy as np

from tmsolve import post
from tmsolve.analysis import process_chain, process_package, solve_chain
from tmsolve.pkgmesh import default_config

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "materials_subset.json")


def test_default_package_chain_steps():
    recs = json.load(open(GOLDEN))
    pkg = process_package(default_config(), recs, "draft")
    steps = process_chain(pkg, recs)
    # S1 with the substrate's Tg (abf_gl 153 and 171 degC) within reach, S2 with the underfill's
    # (111, 112), S3 down to 25 degC; the last step is V11's "S3 30 to 25 degC"
    assert steps[:4] == [(217.0, 187.0, 1), (187.0, 177.0, 1), (177.0, 167.0, 1), (167.0, 165.0, 1)]
    assert steps[4:6] == [(165.0, 155.0, 2), (155.0, 150.0, 2)]
    assert steps[-1] == (30.0, 25.0, 3) and len(steps) == 15
    assert pkg.mesh.ndof == 65322


def test_default_package_rt_warpage(oracle_lib):
    recs = json.load(open(GOLDEN))
    cfg = default_config()
    pkg = process_package(cfg, recs, "draft")
    om = oracle_lib.OracleModel(pkg)
    u, rs = solve_chain(om, pkg, process_chain(pkg, recs))
    assert all(r["converged"] for r in rs)
    b = post.bga_sites(sx=cfg["substrate"]["sx"], sy=cfg["substrate"]["sy"], inset=cfg["bga"]["inset"], pitch=cfg["bga"]["pitch"])
    z = b["zone"]
    w = om.warpage_jeita(u, b["x"], b["y"], [z["x0"], z["x1"], z["y0"], z["y1"]])
    assert f"{1000 * w['signed']:.2f}" == "-69.34", w["signed"]
