"""ctypes wrapper of the CPU oracle (oracle/tm_oracle.cpp) -- TEST INFRASTRUCTURE ONLY.

Imported only by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline
leg, as the checker; the product (libtmsolve.so and the tmsolve package)
never loads it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "libtmoracle.so")

_dp = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
_fp = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_ip = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
_lib = None


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        build()
    L = C.CDLL(LIB_PATH)
    vp = C.c_void_p
    L.orc_model_create.restype = vp
    L.orc_model_create.argtypes = [C.c_int, C.c_int, C.c_int, _dp, _dp, _dp, _ip, _ip, _dp,
                                   C.c_int, _ip, _ip, _ip, _ip, C.c_int, C.c_int, _ip, C.c_double,
                                   C.c_int, _ip, C.c_int, _ip]
    L.orc_model_destroy.argtypes = [vp]
    L.orc_set_module_constraints.argtypes = [vp, C.c_int, _ip]
    L.orc_model_sizes.argtypes = [vp, np.ctypeslib.ndpointer(np.int64, flags="C_CONTIGUOUS")]
    L.orc_model_mesh.argtypes = [vp] + [vp] * 8
    L.orc_assemble.argtypes = [vp, C.c_int, _ip, _dp, _dp, _dp, _dp, _ip, _dp, C.c_int]
    L.orc_get_bcsr.argtypes = [vp, vp, vp, vp, vp]
    L.orc_matvec.argtypes = [vp, _dp, _dp]
    L.orc_solve.restype = C.c_int
    L.orc_solve.argtypes = [vp, _dp, _dp, C.c_double, C.c_int, C.c_int, C.c_long, _dp]
    L.orc_clear_warm.argtypes = [vp]
    L.orc_mg_levels.restype = C.c_int
    L.orc_mg_levels.argtypes = [vp, _ip, C.c_int]
    L.orc_mg_node_agg.restype = C.c_int
    L.orc_mg_node_agg.argtypes = [vp, _ip]
    L.orc_shape_matrices.argtypes = [vp, vp, _dp]
    L.orc_element_k33.argtypes = [C.c_double] * 3 + [_dp, _dp]
    L.orc_element_fth.argtypes = [C.c_double] * 3 + [vp, vp, _dp]
    L.orc_condense33.argtypes = [_dp, vp, _dp, _dp, _dp]
    L.orc_general_element.argtypes = [_dp, _dp, _dp, _dp]
    L.orc_general_derivs.argtypes = [_dp, C.c_double, C.c_double, C.c_double, _dp, _dp, _dp]
    L.orc_anand_step.restype = C.c_double
    L.orc_anand_step.argtypes = [_dp, _dp, _dp, _dp, C.c_double, C.c_double, _dp, _dp, C.c_int, C.c_int]
    L.orc_anand_series_step.restype = C.c_double
    L.orc_anand_series_step.argtypes = [_dp, _dp, _dp, _dp, _dp, C.c_double, _dp, C.c_double, C.c_double, _dp, _dp, C.c_int]
    L.orc_anand_uniaxial.restype = C.c_double
    L.orc_anand_uniaxial.argtypes = [_dp, _dp, C.c_double, C.c_double, C.c_double, C.c_int]
    L.orc_anand_screen.argtypes = [_dp, _dp, _dp, C.c_int, C.c_int, _dp, _dp, C.c_int, _dp, _dp, _ip, _ip, C.c_int,
                                   _dp, _dp, _dp]
    L.orc_anand_screen_pillar.argtypes = [_dp, _dp, _dp, C.c_int, C.c_int, _dp, _dp, C.c_int, _dp, _dp, _ip, _ip, C.c_int,
                                          C.c_double, C.c_double, _dp, _dp, _dp, _dp, _dp]
    L.orc_accumulate_q.argtypes = [vp, _dp, C.c_int, _ip, _dp]
    L.orc_set_sublayers.argtypes = [vp, _ip, _dp, _dp, _dp]
    L.orc_accumulate_state.argtypes = [vp, _dp, C.c_int, _ip, C.c_int, _dp]
    L.orc_state_stress.argtypes = [vp, C.c_int, _ip, _dp, C.c_int, _dp, _dp, _dp]
    L.orc_element_strains.argtypes = [vp, C.c_int, _ip, _dp, _dp, _dp]
    L.orc_fit_plane.argtypes = [C.c_int, _dp, _dp, _dp, _dp]
    L.orc_sample_plane.restype = C.c_double
    L.orc_sample_plane.argtypes = [vp, _dp, C.c_int, C.c_int, C.c_double, C.c_double]
    L.orc_warpage_jeita.argtypes = [vp, _dp, C.c_int, _dp, _dp, _dp, _dp]
    L.orc_pc_apply.argtypes = [vp, _dp, _dp]
    L.orc_sub_create.restype = vp
    L.orc_sub_create.argtypes = [C.c_int, C.c_int, C.c_int, _dp, _dp, _dp, _ip, C.c_int, C.c_int, _dp, _dp, _dp, C.c_int, _ip,
                                 _dp, _dp, _dp, _dp, C.c_int, _dp, _dp, C.c_double, _dp, _dp, _dp, _dp, C.c_double,
                                 C.c_double, C.c_double, C.c_int, C.c_double, C.c_double, C.c_int, _dp, _dp, _dp]
    L.orc_sub_destroy.argtypes = [vp]
    L.orc_sub_elastic.argtypes = [vp, C.c_int, C.c_double, C.c_double, C.c_double, _dp, _dp]
    L.orc_sub_sizes.argtypes = [vp, _ip]
    L.orc_sub_step.argtypes = [vp, C.c_double, C.c_double, _ip, _dp]
    L.orc_sub_get_u.argtypes = [vp, _dp]
    L.orc_sub_get_points.argtypes = [vp, _dp, _dp]
    L.orc_sub_run.argtypes = [vp, C.c_int, _dp, _dp, _ip, _ip, C.c_int, C.c_double, C.c_double, _dp, _dp, _dp, C.c_int, _ip, _dp, _fp]
    L.orc_sub_stress_snapshot.argtypes = [vp, C.c_double, _fp]
    L.orc_last_error.restype = C.c_char_p
    L.orc_last_error.argtypes = [vp]
    _lib = L
    return L


def _ptr(a):
    return a.ctypes.data_as(C.c_void_p) if a is not None else None


class OracleModel:
    """CPU restatement of FEModel + LinearSolver (09-assembly.js, 10-solver.js) on one package."""

    def __init__(self, pkg, constraints=None):
        L = lib()
        m = pkg.mesh
        ncells = (m.nx - 1) * (m.ny - 1) * (m.nz - 1)
        cg = np.full(2 * ncells, -1, np.int32); cp = np.zeros(2 * ncells, np.int32); cs = np.zeros(2 * ncells)
        ce = m.cellElems
        on = ce >= 0
        cg[on] = m.eGroup[ce[on]]; cp[on] = m.ePart[ce[on]]; cs[on] = m.eScale[ce[on]]
        con = np.ascontiguousarray(m.constraints if constraints is None else constraints, np.int32)
        fx = np.ascontiguousarray(m.featureX, np.int32); fy = np.ascontiguousarray(m.featureY, np.int32)
        self.pkg = pkg
        self.h = L.orc_model_create(m.nx, m.ny, m.nz, np.ascontiguousarray(m.xs), np.ascontiguousarray(m.ys),
                                    np.ascontiguousarray(m.zs), cg, cp, cs,
                                    len(pkg.group_layered), np.ascontiguousarray(pkg.group_layered, np.int32),
                                    np.ascontiguousarray(pkg.group_stage, np.int32), np.ascontiguousarray(pkg.group_pset, np.int32),
                                    np.ascontiguousarray(pkg.sec_of_layer, np.int32), int(pkg.npset),
                                    len(con), con, 0.0, len(fx), fx if len(fx) else np.zeros(1, np.int32),
                                    len(fy), fy if len(fy) else np.zeros(1, np.int32))
        mc = getattr(m, "moduleConstraints", None)
        if mc is not None and len(mc):
            L.orc_set_module_constraints(self.h, len(mc), np.ascontiguousarray(mc, np.int32))
        sz = np.zeros(5, np.int64)
        L.orc_model_sizes(self.h, sz)
        self.nn, self.ne, self.nb, self.ndof, self.ncon = (int(v) for v in sz)

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_model_destroy(self.h)
            self.h = None

    def mesh_arrays(self):
        m = self.pkg.mesh
        out = dict(nodeId=np.zeros(m.nx * m.ny * m.nz, np.int32), conn=np.zeros(8 * self.ne, np.int32),
                   eIJK=np.zeros(3 * self.ne, np.int32), colStart=np.zeros(m.nx * m.ny + 1, np.int32),
                   cellElems=np.zeros(2 * (m.nx - 1) * (m.ny - 1) * (m.nz - 1), np.int32),
                   coords=np.zeros(3 * self.nn), constraints=np.zeros(self.ncon, np.int32), eGroup=np.zeros(self.ne, np.int32))
        lib().orc_model_mesh(self.h, *[_ptr(out[k]) for k in ("nodeId", "conn", "eIJK", "colStart", "cellElems", "coords", "constraints", "eGroup")])
        return out

    def assemble(self, step, no_constraints=False):
        rhs = np.zeros(self.ndof)
        lib().orc_assemble(self.h, int(step.stage), np.ascontiguousarray(step.layered, np.int32), step.D, step.s0, step.W, step.V,
                           np.ascontiguousarray(step.born, np.int32), rhs, int(no_constraints))
        return rhs

    def prepare_step(self, step):
        """The step's shape matrices and thermal loads for the DOF histories (an assembly here)."""
        self.assemble(step)

    def bcsr(self):
        rowPtr = np.zeros(self.nn + 1, np.int32); col = np.zeros(self.nb, np.int32)
        val = np.zeros(9 * self.nb); isC = np.zeros(self.ndof, np.uint8)
        lib().orc_get_bcsr(self.h, _ptr(rowPtr), _ptr(col), _ptr(val), _ptr(isC))
        return rowPtr, col, val, isC

    def matvec(self, x):
        y = np.zeros(self.ndof)
        lib().orc_matvec(self.h, np.ascontiguousarray(x, np.float64), y)
        return y

    def solve(self, f, tol=1e-8, maxit=2000, precond="mg", key=-1):
        """LinearSolver.solve (10-solver.js:933-994). The assembled values are scaled in place."""
        u = np.zeros(self.ndof)
        info = np.zeros(16)
        rc = lib().orc_solve(self.h, np.ascontiguousarray(f, np.float64), u, float(tol), int(maxit),
                             0 if precond == "mg" else 1, int(key), info)
        if rc:
            raise RuntimeError(lib().orc_last_error(self.h).decode())
        keys = ["iters", "relres", "converged", "iters0", "ms", "pcMs", "precond", "rebuilt", "warm", "fallback",
                "colJitter", "shellJitter", "levels"]
        rec = {k: float(info[i]) for i, k in enumerate(keys)}
        for k in ("iters", "converged", "rebuilt", "warm", "fallback", "colJitter", "shellJitter", "levels"):
            rec[k] = int(rec[k])
        rec["precond"] = "mg" if info[6] == 0 else "ic"
        rec["u"] = u
        return rec

    def pc_apply(self, r):
        """pc.apply of the preconditioner the last solve built (scaled space)."""
        z = np.zeros(self.ndof)
        if lib().orc_pc_apply(self.h, np.ascontiguousarray(r, np.float64), z):
            raise RuntimeError("no preconditioner built")
        return z

    def clear_warm(self):
        lib().orc_clear_warm(self.h)

    def mg_levels(self):
        out = np.zeros(4 * 64, np.int32)
        n = lib().orc_mg_levels(self.h, out, 64)
        return [tuple(out[4 * l:4 * l + 4]) for l in range(n)]

    def mg_node_agg(self):
        out = np.zeros(self.nn, np.int32)
        lib().orc_mg_node_agg(self.h, out)
        return out

    def accumulate_q(self, du, elems, q):
        """Model.accumulateStep with qOnly (09-assembly.js:508-533) of the last assembled step:
        q (nel x 33, updated in place) += the DOF increment of every element of elems."""
        elems = np.ascontiguousarray(elems, np.int32)
        assert q.dtype == np.float64 and q.flags.c_contiguous and q.size == 33 * len(elems)
        lib().orc_accumulate_q(self.h, np.ascontiguousarray(du, np.float64), len(elems), elems, q)
        return q

    def set_sublayers(self, step):
        """The step's sub-layers of the layered property sets (for the stress histories)."""
        f = lambda a: np.ascontiguousarray(a if a is not None and len(a) else np.zeros(1), np.float64)
        lib().orc_set_sublayers(self.h, np.ascontiguousarray(step.sub_n, np.int32), f(step.sub_z), f(step.sub_D), f(step.sub_s0))

    def accumulate_state(self, du, elems, stride, state):
        """Model.accumulateStep (09-assembly.js:508-544) of the last assembled step: state (nel x
        stride) += the DOF increment and the sub-layer stress monomials."""
        elems = np.ascontiguousarray(elems, np.int32)
        assert state.dtype == np.float64 and state.flags.c_contiguous and state.size == stride * len(elems)
        lib().orc_accumulate_state(self.h, np.ascontiguousarray(du, np.float64), len(elems), elems, int(stride), state)
        return state

    def state_stress(self, elem, state, stride, nat):
        """stateStress (09-assembly.js:555-571): (eps, sig), each (npts, 6)."""
        elem = np.ascontiguousarray(elem, np.int32)
        eps = np.zeros(6 * len(elem)); sig = np.zeros(6 * len(elem))
        lib().orc_state_stress(self.h, len(elem), elem, np.ascontiguousarray(state, np.float64).reshape(-1), int(stride),
                               np.ascontiguousarray(nat, np.float64).reshape(-1), eps, sig)
        return eps.reshape(-1, 6), sig.reshape(-1, 6)

    def element_strains(self, elem, q, nat):
        """boxStrainAt (07-element.js:127-142) of element elem[t] with DOFs q[t] at nat[t]."""
        elem = np.ascontiguousarray(elem, np.int32)
        eps = np.zeros(6 * len(elem))
        lib().orc_element_strains(self.h, len(elem), elem, np.ascontiguousarray(q, np.float64).reshape(-1),
                                  np.ascontiguousarray(nat, np.float64).reshape(-1), eps)
        return eps.reshape(-1, 6)

    def sample_plane(self, u, k, comp, x, y):
        return lib().orc_sample_plane(self.h, np.ascontiguousarray(u, np.float64), int(k), int(comp), float(x), float(y))

    def warpage_jeita(self, u, bx, by, zone):
        """warpageJEITA (12-post.js:60-109): dict of signed, mag, sign, signConf, plane, rmin, rmax."""
        out = np.zeros(9)
        bx = np.ascontiguousarray(bx, np.float64); by = np.ascontiguousarray(by, np.float64)
        lib().orc_warpage_jeita(self.h, np.ascontiguousarray(u, np.float64), len(bx), bx, by,
                                np.ascontiguousarray(zone, np.float64), out)
        return dict(signed=out[0], mag=out[1], sign=out[2], signConf=out[3], plane=out[4:7].copy(), rmin=out[7], rmax=out[8])


def fit_plane(x, y, w):
    c = np.zeros(3)
    lib().orc_fit_plane(len(w), np.ascontiguousarray(x, np.float64), np.ascontiguousarray(y, np.float64),
                        np.ascontiguousarray(w, np.float64), c)
    return c


def anand_series_step(params, Etab, state, eps, tz, fs, Cp, T, dt, commit=True):
    """stepSeriesColumn of one point: (plastic increment, sig, D); eps (the cap's strain) and
    state are updated in place."""
    sig = np.zeros(6); D = np.zeros(36)
    d = lib().orc_anand_series_step(np.ascontiguousarray(params, np.float64), np.ascontiguousarray(Etab, np.float64), state, eps,
                                    np.ascontiguousarray(tz, np.float64), float(fs), np.ascontiguousarray(Cp, np.float64),
                                    float(T), float(dt), sig, D, int(commit))
    return d, sig, D


def anand_uniaxial(params, Etab, T, rate, eps_max, nsteps):
    return lib().orc_anand_uniaxial(np.ascontiguousarray(params, np.float64), np.ascontiguousarray(Etab, np.float64),
                                    float(T), float(rate), float(eps_max), int(nsteps))


def anand_step(params, Etab, state, eps, T, dt, want_tangent=True, commit=True):
    sig = np.zeros(6); D = np.zeros(36)
    d = lib().orc_anand_step(np.ascontiguousarray(params, np.float64), np.ascontiguousarray(Etab, np.float64), state,
                             np.ascontiguousarray(eps, np.float64), float(T), float(dt), sig, D, int(want_tangent), int(commit))
    return d, sig, D


def anand_screen(params, Etab, Ftab, temps, table, hist):
    """screenJoints' per-site loop (13-fatigue.js:395-451) for free-standing solder columns."""
    temps = np.ascontiguousarray(temps, np.float64); table = np.ascontiguousarray(table, np.float64)
    nsites = table.size // (6 * len(temps))
    dW = np.zeros(nsites); dE = np.zeros(nsites); stab = np.zeros(nsites)
    lib().orc_anand_screen(np.ascontiguousarray(params, np.float64), np.ascontiguousarray(Etab, np.float64),
                           np.ascontiguousarray(Ftab, np.float64), nsites, len(temps), temps, table,
                           len(hist["t"]), np.ascontiguousarray(hist["t"], np.float64), np.ascontiguousarray(hist["T"], np.float64),
                           np.ascontiguousarray(hist["cycle"], np.int32), np.ascontiguousarray(hist["phase"], np.int32),
                           int(hist["cycles"]), dW, dE, stab)
    return dW, dE, stab


def anand_screen_pillar(params, Etab, Ftab, temps, table, hist, fs, pnu, pEtab, pFtab):
    """screenJoints' per-site loop for a solder cap (height fraction fs) on an elastic pillar
    (stepSeriesColumn, 13-fatigue.js:178-206, as screenDdi drives it, :369-376)."""
    temps = np.ascontiguousarray(temps, np.float64); table = np.ascontiguousarray(table, np.float64)
    nsites = table.size // (6 * len(temps))
    dW = np.zeros(nsites); dE = np.zeros(nsites); stab = np.zeros(nsites)
    lib().orc_anand_screen_pillar(np.ascontiguousarray(params, np.float64), np.ascontiguousarray(Etab, np.float64),
                                  np.ascontiguousarray(Ftab, np.float64), nsites, len(temps), temps, table,
                                  len(hist["t"]), np.ascontiguousarray(hist["t"], np.float64),
                                  np.ascontiguousarray(hist["T"], np.float64), np.ascontiguousarray(hist["cycle"], np.int32),
                                  np.ascontiguousarray(hist["phase"], np.int32), int(hist["cycles"]), float(fs), float(pnu),
                                  np.ascontiguousarray(pEtab, np.float64), np.ascontiguousarray(pFtab, np.float64), dW, dE, stab)
    return dW, dE, stab


class OracleSubmodel:
    """CPU restatement of BumpSubmodel (13-fatigue.js:470-1104) on a SubmodelSpec."""

    def __init__(self, spec):
        L = lib()
        f = lambda a: np.ascontiguousarray(a, np.float64)
        i32 = lambda a: np.ascontiguousarray(a, np.int32)
        self._keep = (f(spec.xs), f(spec.ys), f(spec.zs))
        nb = len(spec.bGlob)
        self.h = L.orc_sub_create(len(spec.xs), len(spec.ys), len(spec.zs), f(spec.xs), f(spec.ys), f(spec.zs), i32(spec.cell_mat),
                                  spec.nglob, len(spec.ts), f(spec.ts), f(spec.fields), f(spec.u25), nb, i32(spec.bGlob).reshape(-1),
                                  f(spec.bW).reshape(-1), f(spec.anand), f(spec.solder_E), f(spec.solder_F), int(spec.elastic_solder),
                                  f(spec.uf_E), f(spec.uf_F), float(spec.uf_nu), f(spec.si_D), f(spec.si_F), f(spec.sub_D),
                                  f(spec.sub_F), float(spec.nu_max), float(spec.zt), float(spec.zaf), int(spec.uniform),
                                  float(spec.density), float(spec.nu_max_global), spec.nsec, *spec.section_arrays())
        if not self.h:
            raise ValueError("boundary node count does not match the cell")
        sz = np.zeros(4, np.int32)
        L.orc_sub_sizes(self.h, sz)
        self.nn, self.ne, self.nb, self.nsolder = (int(v) for v in sz)
        self.ndof = 3 * self.nn

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_sub_destroy(self.h)
            self.h = None

    def elastic(self, mat, Ta, Tb, sub_z=0.0):
        """_elastic (13-fatigue.js:702-757) of material mat (0 substrate, 1 solder, 2 underfill,
        3 silicon) over the step from Ta to Tb: (D 36, thermal stress increment 6)."""
        D, sth = np.zeros(36), np.zeros(6)
        lib().orc_sub_elastic(self.h, int(mat), float(sub_z), float(Ta), float(Tb), D, sth)
        return D, sth

    def step(self, T, dt):
        """stepTo (13-fatigue.js:924-956): (converged, newton, dMax)."""
        nw = np.zeros(1, np.int32); dm = np.zeros(1)
        ok = lib().orc_sub_step(self.h, float(T), float(dt), nw, dm)
        return bool(ok), int(nw[0]), float(dm[0])

    def u(self):
        out = np.zeros(self.ndof)
        lib().orc_sub_get_u(self.h, out)
        return out

    def points(self):
        W = np.zeros(self.nsolder); E = np.zeros(self.nsolder)
        lib().orc_sub_get_points(self.h, W, E)
        return W, E

    def run(self, hist, cphi=1.0, sphi=0.0, max_snaps=0):
        """run (13-fatigue.js:1004-1104): dict of dW, dWdie, dWsub, dE, dEdie, dEsub, stabChange,
        steps, cutbacks, newtonPerStep, perCycle (cycles x 2), loop (points x 4); with max_snaps,
        the stress snapshots of the last cycle: snaps_meta (T, t, cycle, phase) and snaps
        (float32, n x ne x 8 x 6)."""
        n, nc = len(hist["t"]), int(hist["cycles"])
        out = np.zeros(10); pc = np.zeros(2 * nc); loop = np.zeros(4 * n)
        ns = np.zeros(1, np.int32); meta = np.zeros(4 * max(max_snaps, 1)); sig = np.zeros(48 * self.ne * max(max_snaps, 1), np.float32)
        rc = lib().orc_sub_run(self.h, n, np.ascontiguousarray(hist["t"], np.float64), np.ascontiguousarray(hist["T"], np.float64),
                               np.ascontiguousarray(hist["cycle"], np.int32), np.ascontiguousarray(hist["phase"], np.int32), nc,
                               float(cphi), float(sphi), out, pc, loop, int(max_snaps), ns, meta, sig)
        if rc:
            raise RuntimeError("submodel run failed")
        keys = ["dW", "dWdie", "dWsub", "dE", "dEdie", "dEsub", "stabChange", "steps", "cutbacks", "newtonPerStep"]
        rec = {k: float(out[i]) for i, k in enumerate(keys)}
        rec["perCycle"] = pc.reshape(nc, 2); rec["loop"] = loop.reshape(n, 4)
        k = min(int(ns[0]), max_snaps)
        rec["nsnaps"] = int(ns[0])
        rec["snaps_meta"] = meta[:4 * k].reshape(k, 4); rec["snaps"] = sig[:48 * self.ne * k].reshape(k, self.ne, 8, 6)
        return rec

    def stress_snapshot(self, T):
        """_stressSnapshot (13-fatigue.js:965-989) of the current state: float32 (ne, 8, 6)."""
        out = np.zeros(48 * self.ne, np.float32)
        lib().orc_sub_stress_snapshot(self.h, float(T), out)
        return out.reshape(self.ne, 8, 6)

