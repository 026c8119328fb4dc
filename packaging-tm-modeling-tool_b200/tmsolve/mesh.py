"""Structured extruded hex mesh -- the host-side form of the tool's mesher output.

The reference's mesher stays on the caller's side of the boundary; this module
builds the same arrays from grid lines and a cell assignment so that the
library can be driven without it. Node and element numbering is the bit-exact
contract of the boundary:

* ``buildStructuredMesh`` (src/core/06-mesher.js:14-72): elements in cell order
  (i, j, k) with k fastest, up to two superposed phases per cell; nodes exist
  only where attached to an element and are numbered z fastest, then y, then x;
  local node order ``loc`` (06-mesher.js:49); column c = i*ny + j holds the
  contiguous node range colStart[c] .. colStart[c+1]-1.
* ``constraints321`` (06-mesher.js:112-116) with ``nearestNodeOnPlane`` (:75-84).
* ``module_support`` (``moduleSupport``, 06-mesher.js:92-109): the three support nodes of a
  stacked module on its base bottom plane.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

LOC = np.array([[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0],
                [0, 0, 1], [1, 0, 1], [1, 1, 1], [0, 1, 1]], dtype=np.int64)

# part ids of 06-mesher.js:3-4
PART = dict(SUB=0, SOLDER=1, UF_BUMP=2, UF_FILLET=3, DIE=4, TIM=5, LID=6, LIDADH=7, STIFF=8, STIFFADH=9,
            CHIPLET=10, BASE_SI=11, TSV=12, RDL=13, DDI_SOLDER=14, DDI_FILL=15, WCUF_FILLET=16, MOLD=17)


@dataclass
class Mesh:
    xs: np.ndarray
    ys: np.ndarray
    zs: np.ndarray
    nx: int
    ny: int
    nz: int
    nn: int
    ne: int
    coords: np.ndarray       # (nn*3,) float64
    nodeIJK: np.ndarray      # (nn*3,) int32
    nodeId: np.ndarray       # (nx*ny*nz,) int32, -1 where absent
    conn: np.ndarray         # (ne*8,) int32
    eIJK: np.ndarray         # (ne*3,) int32
    colStart: np.ndarray     # (nx*ny+1,) int32
    cellElems: np.ndarray    # (ncells*2,) int32
    eGroup: np.ndarray       # (ne,) int32
    ePart: np.ndarray        # (ne,) int8
    eScale: np.ndarray       # (ne,) float64
    featureX: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int32))
    featureY: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int32))
    constraints: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int32))
    # stacked modules: each module's 3-2-1 support DOFs on its base bottom (mesh.moduleConstraints,
    # 06-mesher.js:535-545), None for a package without modules
    moduleConstraints: np.ndarray = None

    @property
    def ndof(self) -> int:
        return 3 * self.nn


def pack_cells(cell_group: np.ndarray, cell_part: np.ndarray, cell_scale: np.ndarray):
    """Move the phases of every cell to the front (the reference fills cellElems[2c+q] in list order)."""
    g = np.asarray(cell_group, np.int32).reshape(-1, 2).copy()
    p = np.asarray(cell_part, np.int32).reshape(-1, 2).copy()
    s = np.asarray(cell_scale, np.float64).reshape(-1, 2).copy()
    swap = (g[:, 0] < 0) & (g[:, 1] >= 0)
    for a in (g, p, s):
        a[swap] = a[swap][:, ::-1]
    return g.ravel(), p.ravel(), s.ravel()


def build_structured_mesh(xs, ys, zs, cell_group, cell_part, cell_scale, featureX=None, featureY=None) -> Mesh:
    """buildStructuredMesh (06-mesher.js:14-72) from per-cell phase arrays of length 2*ncells.

    cell_group[2c+q] < 0 marks no element; cells are indexed c = (i*(ny-1) + j)*(nz-1) + k.
    """
    xs = np.asarray(xs, np.float64); ys = np.asarray(ys, np.float64); zs = np.asarray(zs, np.float64)
    nx, ny, nz = len(xs), len(ys), len(zs)
    ncy, ncz = ny - 1, nz - 1
    ncells = (nx - 1) * ncy * ncz
    g, p, s = pack_cells(cell_group, cell_part, cell_scale)
    if g.size != 2 * ncells:
        raise ValueError("cell arrays must hold 2 entries per cell")
    slots = np.nonzero(g >= 0)[0]                 # cell then phase order
    ne = int(slots.size)
    eCell = (slots // 2).astype(np.int64)
    cellElems = np.full(2 * ncells, -1, np.int32)
    cellElems[slots] = np.arange(ne, dtype=np.int32)
    k = eCell % ncz
    j = (eCell // ncz) % ncy
    i = eCell // (ncz * ncy)
    exist = np.zeros(nx * ny * nz, np.uint8)
    for a in range(8):
        exist[((i + LOC[a, 0]) * ny + j + LOC[a, 1]) * nz + k + LOC[a, 2]] = 1
    nodeId = np.full(nx * ny * nz, -1, np.int32)
    on = np.nonzero(exist)[0]
    nn = int(on.size)
    nodeId[on] = np.arange(nn, dtype=np.int32)
    ni = on // (ny * nz)
    nj = (on // nz) % ny
    nk = on % nz
    coords = np.empty(nn * 3, np.float64)
    coords[0::3] = xs[ni]; coords[1::3] = ys[nj]; coords[2::3] = zs[nk]
    nodeIJK = np.empty(nn * 3, np.int32)
    nodeIJK[0::3] = ni; nodeIJK[1::3] = nj; nodeIJK[2::3] = nk
    conn = np.empty((ne, 8), np.int32)
    for a in range(8):
        conn[:, a] = nodeId[((i + LOC[a, 0]) * ny + j + LOC[a, 1]) * nz + k + LOC[a, 2]]
    eIJK = np.stack([i, j, k], axis=1).astype(np.int32).ravel()
    per_col = (nodeId.reshape(nx * ny, nz) >= 0).sum(axis=1)
    colStart = np.zeros(nx * ny + 1, np.int32)
    colStart[1:] = np.cumsum(per_col)
    return Mesh(xs=xs, ys=ys, zs=zs, nx=nx, ny=ny, nz=nz, nn=nn, ne=ne, coords=coords, nodeIJK=nodeIJK,
                nodeId=nodeId, conn=conn.ravel(), eIJK=eIJK, colStart=colStart, cellElems=cellElems,
                eGroup=g[slots].astype(np.int32), ePart=p[slots].astype(np.int8), eScale=s[slots].astype(np.float64),
                featureX=np.asarray(featureX if featureX is not None else [], np.int32),
                featureY=np.asarray(featureY if featureY is not None else [], np.int32))


def nearest_node_on_plane(mesh: Mesh, x: float, y: float, k: int) -> int:
    """nearestNodeOnPlane (06-mesher.js:75-84): first node in (i, j) order within 1e-12 of the minimum distance."""
    best, bd = -1, np.inf
    for i in range(mesh.nx):
        for j in range(mesh.ny):
            nid = int(mesh.nodeId[(i * mesh.ny + j) * mesh.nz + k])
            if nid < 0:
                continue
            d = float(np.hypot(mesh.xs[i] - x, mesh.ys[j] - y))
            if d < bd - 1e-12:
                bd, best = d, nid
    return best


def constraints321(mesh: Mesh, a: float) -> np.ndarray:
    """constraints321 (06-mesher.js:112-116): 3-2-1 rigid-body DOFs on the bottom plane."""
    n0 = nearest_node_on_plane(mesh, 0.0, 0.0, 0)
    n1 = nearest_node_on_plane(mesh, a, 0.0, 0)
    n2 = nearest_node_on_plane(mesh, 0.0, a, 0)
    return np.array([3 * n0, 3 * n0 + 1, 3 * n0 + 2, 3 * n1 + 1, 3 * n1 + 2, 3 * n2 + 2], np.int32)


def module_support(mesh: Mesh, rect: dict, cx: float, cy: float, k: int):
    """moduleSupport (06-mesher.js:92-109): three nodes of plane k inside rect (x0, x1, y0, y1):
    a the nearest to (cx, cy), b on a's row farthest from it in x, c off that row, farthest in y
    (ties to the smaller x distance); None when there are too few."""
    tol = 1e-9
    cand = []
    for i in range(mesh.nx):
        x = float(mesh.xs[i])
        if x < rect["x0"] - tol or x > rect["x1"] + tol:
            continue
        for j in range(mesh.ny):
            y = float(mesh.ys[j])
            nid = int(mesh.nodeId[(i * mesh.ny + j) * mesh.nz + k])
            if nid >= 0 and rect["y0"] - tol <= y <= rect["y1"] + tol:
                cand.append((nid, x, y))
    if len(cand) < 3:
        return None

    def pick(score, ok):
        best, bs = None, -math.inf
        for c in cand:
            if ok(c):
                s = score(c)
                if s > bs + tol:
                    bs, best = s, c
        return best
    a = pick(lambda c: -math.hypot(c[1] - cx, c[2] - cy), lambda c: True)
    b = pick(lambda c: abs(c[1] - a[1]), lambda c: abs(c[2] - a[2]) < tol and c[0] != a[0])
    if b is None:
        return None
    c = pick(lambda c: abs(c[2] - a[2]) - 1e-6 * abs(c[1] - a[1]), lambda c: abs(c[2] - a[2]) > tol)
    return None if c is None else [a[0], b[0], c[0]]
