"""Host-side mesher mirror against the oracle's restatement of buildStructuredMesh
(06-mesher.js:14-72) and constraints321 (:112-116): node, element and DOF indexing is
the bit-exact contract of the boundary."""
import numpy as np
import pytest

from tmsolve.packages import box_package, fcbga_c1, lidded_c2, linspace
from tmsolve.materials import iso_d


def _compare(pkg, oracle_lib):
    om = oracle_lib.OracleModel(pkg)
    o = om.mesh_arrays()
    m = pkg.mesh
    assert om.nn == m.nn and om.ne == m.ne
    for k in ("nodeId", "conn", "eIJK", "colStart", "cellElems", "eGroup"):
        assert np.array_equal(o[k], getattr(m, k)), k
    assert np.array_equal(o["coords"], m.coords)
    assert np.array_equal(o["constraints"], m.constraints)


def test_c1_indexing(oracle_lib):
    pkg = fcbga_c1()
    assert (pkg.mesh.nn, pkg.mesh.ne) == (32661, 29952)
    _compare(pkg, oracle_lib)


def test_c2_small_indexing(oracle_lib):
    _compare(lidded_c2(n_inplane=32), oracle_lib)


def test_box_with_voids_indexing(oracle_lib):
    mats = [(iso_d(1000.0, 0.3), 1e-5, 1e-5)]
    pkg = box_package(linspace(0, 3, 3), linspace(0, 2, 2), linspace(0, 1, 4), mats,
                      lambda i, j, k: 0 if (k < 2 or (i == 1 and j == 0)) else -1)
    _compare(pkg, oracle_lib)


def test_superposed_phases_packed():
    pkg = fcbga_c1()
    m = pkg.mesh
    ce = m.cellElems.reshape(-1, 2)
    # second phase only where a first exists, and phases in element order
    assert not np.any((ce[:, 0] < 0) & (ce[:, 1] >= 0))
    both = ce[:, 1] >= 0
    assert np.all(ce[both, 1] == ce[both, 0] + 1)
    assert set(np.unique(m.ePart[ce[both, 0]])) == {1} and set(np.unique(m.ePart[ce[both, 1]])) == {2}
