"""Host-side mirror of the reference's solver interface over the GPU C-ABI.

``DeviceModel`` stands for ``FEModel`` + ``LinearSolver`` of the reference
(src/core/09-assembly.js:208, src/core/10-solver.js:826):

* ``assemble_step(step)``  ->  ``FEModel.assembleStep(Ta, Tb, stage, rhs)``: the per-step
  property sets are computed by the caller (``prepareStep``'s output) and the assembly,
  condensation and constraints run on the GPU;
* ``set_bcsr(...)``        ->  solving a caller-assembled ``model.pattern``/``model.val``;
* ``solve(f, label, key)`` ->  ``LinearSolver.solve``: returns the reference's record
  ``{u, iters, relres, converged, ms, pcMs, precond, rebuilt, warm, iters0, fallback}``;
  non-convergence gives ``converged: False`` (the caller decides to throw, as
  ``Analysis.solveStep`` does, src/core/11-analysis.js:204); every other failure raises.
"""
from __future__ import annotations

import ctypes as C
from typing import Optional

import numpy as np

from . import _lib
from ._lib import TmError, TmMesh, TmSolveInfo, TmSolveOpts, TmStep, check, load
from .packages import Package, StepData


def _p(a, ctype):
    return a.ctypes.data_as(C.POINTER(ctype)) if a is not None else None


def _out_array(out, n):
    if out is None:
        return np.zeros(n)
    if out.dtype != np.float64 or out.shape != (n,) or not out.flags.c_contiguous:
        raise ValueError(f"out must be a contiguous float64 array of {n} values")
    return out


class DeviceModel:
    def __init__(self, pkg: Package, constraints: Optional[np.ndarray] = None):
        L = load()
        m = pkg.mesh
        self.pkg = pkg
        self._keep = []

        def keep(a, dtype):
            a = np.ascontiguousarray(a, dtype)
            self._keep.append(a)
            return a

        xs, ys, zs = keep(m.xs, np.float64), keep(m.ys, np.float64), keep(m.zs, np.float64)
        con = keep(m.constraints if constraints is None else constraints, np.int32)
        fx = keep(m.featureX, np.int32); fy = keep(m.featureY, np.int32)
        mc = keep(getattr(m, "moduleConstraints", None) if getattr(m, "moduleConstraints", None) is not None else [], np.int32)
        mesh = TmMesh(nx=m.nx, ny=m.ny, nz=m.nz, xs=_p(xs, C.c_double), ys=_p(ys, C.c_double), zs=_p(zs, C.c_double),
                      nn=m.nn, ne=m.ne, coords=_p(keep(m.coords, np.float64), C.c_double),
                      nodeId=_p(keep(m.nodeId, np.int32), C.c_int32), conn=_p(keep(m.conn, np.int32), C.c_int32),
                      eIJK=_p(keep(m.eIJK, np.int32), C.c_int32), colStart=_p(keep(m.colStart, np.int32), C.c_int32),
                      cellElems=_p(keep(m.cellElems, np.int32), C.c_int32), eGroup=_p(keep(m.eGroup, np.int32), C.c_int32),
                      ePart=_p(keep(m.ePart, np.int8), C.c_int8), eScale=_p(keep(m.eScale, np.float64), C.c_double),
                      ngroups=len(pkg.group_stage), groupStage=_p(keep(pkg.group_stage, np.int32), C.c_int32),
                      npset=int(pkg.npset), ePset=_p(keep(pkg.e_pset, np.int32), C.c_int32),
                      nconstr=len(con), constr=_p(con, C.c_int32), nfeatureX=len(fx), nfeatureY=len(fy),
                      featureX=_p(fx, C.c_int32) if len(fx) else None, featureY=_p(fy, C.c_int32) if len(fy) else None,
                      nmodconstr=len(mc), modconstr=_p(mc, C.c_int32) if len(mc) else None)
        h = C.c_void_p()
        check(L.tm_create(C.byref(mesh), C.byref(h)))
        self.h = h
        self._keep = []
        self.ndof = 3 * m.nn
        sz = (C.c_int64 * 6)()
        check(L.tm_sizes(self.h, sz))
        self.nn, self.ne, self.nb, _, self.levels, self.coarsest_dof = (int(v) for v in sz)
        self.log = []

    def close(self):
        if getattr(self, "h", None):
            load().tm_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---- FEModel.assembleStep ------------------------------------------------------------
    @staticmethod
    def _step_struct(step: StepData):
        """tm_step over the step's arrays; the arrays are returned too, to keep them alive."""
        keep = (np.ascontiguousarray(step.layered, np.int32), np.ascontiguousarray(step.born, np.int32),
                np.ascontiguousarray(step.D, np.float64), np.ascontiguousarray(step.s0, np.float64),
                np.ascontiguousarray(step.W, np.float64), np.ascontiguousarray(step.V, np.float64))
        lay, born, D, s0, W, V = keep
        st = TmStep(stage=int(step.stage), psetLayered=_p(lay, C.c_int32), D=_p(D, C.c_double), s0=_p(s0, C.c_double),
                    W=_p(W, C.c_double), V=_p(V, C.c_double), psetBorn=_p(born, C.c_int32))
        return st, keep

    def assemble_step(self, step: StepData, out: Optional[np.ndarray] = None) -> np.ndarray:
        """The load vector of the step (host array; `out`, e.g. pinned memory, is filled when given)."""
        st, _keep = self._step_struct(step)
        rhs = _out_array(out, self.ndof)
        check(load().tm_assemble_step(self.h, C.byref(st), rhs.ctypes.data_as(C.c_void_p)))
        return rhs

    def assemble_step_device(self, step: StepData, rhs_ptr: int):
        """assemble_step with the load written to device memory (raw device pointer)."""
        st, _keep = self._step_struct(step)
        check(load().tm_assemble_step_device(self.h, C.byref(st), C.c_void_p(rhs_ptr)))

    def prepare_step(self, step: StepData):
        """FEModel.stepRecovery (src/core/09-assembly.js:480-491): loads the step's shape matrices
        and element thermal loads for accumulate_q without assembling the operator."""
        st, _keep = self._step_struct(step)
        check(load().tm_prepare_step(self.h, C.byref(st)))

    def set_bcsr(self, rowPtr, col, val, isConstrained):
        rowPtr = np.ascontiguousarray(rowPtr, np.int32); col = np.ascontiguousarray(col, np.int32)
        val = np.ascontiguousarray(val, np.float64); isC = np.ascontiguousarray(isConstrained, np.uint8)
        check(load().tm_set_bcsr(self.h, rowPtr.ctypes.data_as(C.c_void_p), col.ctypes.data_as(C.c_void_p),
                                 val.ctypes.data_as(C.c_void_p), isC.ctypes.data_as(C.c_void_p)))

    def get_bcsr(self):
        rowPtr = np.zeros(self.nn + 1, np.int32); col = np.zeros(self.nb, np.int32); val = np.zeros(9 * self.nb)
        check(load().tm_get_bcsr(self.h, rowPtr.ctypes.data_as(C.c_void_p), col.ctypes.data_as(C.c_void_p),
                                 val.ctypes.data_as(C.c_void_p)))
        return rowPtr, col, val

    def matvec(self, x) -> np.ndarray:
        x = np.ascontiguousarray(x, np.float64)
        y = np.zeros(self.ndof)
        check(load().tm_matvec(self.h, x.ctypes.data_as(C.c_void_p), y.ctypes.data_as(C.c_void_p)))
        return y

    # ---- element DOF histories and field sampling ------------------------------------------
    def accumulate_q(self, du, elems, q: np.ndarray) -> np.ndarray:
        """Model.accumulateStep with qOnly (src/core/09-assembly.js:508-533) for the step
        assembled last: q (nel x 33, float64, updated in place) += every listed element's DOF
        increment from the step's displacement increment du. A negative element index (no
        element at that site) gives a NaN row."""
        du = np.ascontiguousarray(du, np.float64); elems = np.ascontiguousarray(elems, np.int32)
        if q.dtype != np.float64 or not q.flags.c_contiguous or q.size != 33 * len(elems):
            raise ValueError("q must be a contiguous float64 array of 33 values per element")
        if du.size != self.ndof:
            raise ValueError(f"du must hold {self.ndof} values")
        check(load().tm_accumulate_q(self.h, du.ctypes.data_as(C.c_void_p), len(elems), elems.ctypes.data_as(C.c_void_p),
                                     q.ctypes.data_as(C.c_void_p)))
        return q

    def element_strains(self, elem, q, nat) -> np.ndarray:
        """boxStrainAt (src/core/07-element.js:127-142) of element elem[p] with DOFs q[p] at the
        natural point nat[p]: (npts, 6) engineering strains."""
        elem = np.ascontiguousarray(elem, np.int32)
        q = np.ascontiguousarray(q, np.float64).reshape(-1); nat = np.ascontiguousarray(nat, np.float64).reshape(-1)
        if q.size != 33 * len(elem) or nat.size != 3 * len(elem):
            raise ValueError("q needs 33 and nat 3 values per point")
        eps = np.zeros(6 * len(elem))
        check(load().tm_element_strains(self.h, len(elem), elem.ctypes.data_as(C.c_void_p), q.ctypes.data_as(C.c_void_p),
                                        nat.ctypes.data_as(C.c_void_p), eps.ctypes.data_as(C.c_void_p)))
        return eps.reshape(-1, 6)

    def element_strains_adjoint(self, elem, nat, g) -> np.ndarray:
        """The transpose of element_strains: (npts, 33) B^T g for strain derivatives g (npts, 6)."""
        elem = np.ascontiguousarray(elem, np.int32)
        nat = np.ascontiguousarray(nat, np.float64).reshape(-1); g = np.ascontiguousarray(g, np.float64).reshape(-1)
        if nat.size != 3 * len(elem) or g.size != 6 * len(elem):
            raise ValueError("nat needs 3 and g 6 values per point")
        gq = np.zeros(33 * len(elem))
        vp = lambda a: a.ctypes.data_as(C.c_void_p)
        check(load().tm_element_strains_adjoint(self.h, len(elem), vp(elem), vp(nat), vp(g), vp(gq)))
        return gq.reshape(-1, 33)

    def accumulate_q_adjoint(self, elems, gq):
        """The transpose of one accumulate_q step (the step loaded last): (gdu (nel, 24), gA (nel,))."""
        elems = np.ascontiguousarray(elems, np.int32)
        gq = np.ascontiguousarray(gq, np.float64).reshape(-1)
        if gq.size != 33 * len(elems):
            raise ValueError("gq needs 33 values per element")
        gdu = np.zeros(24 * len(elems)); gA = np.zeros(len(elems))
        vp = lambda a: a.ctypes.data_as(C.c_void_p)
        check(load().tm_accumulate_q_adjoint(self.h, len(elems), vp(elems), vp(gq), vp(gdu), vp(gA)))
        return gdu.reshape(-1, 24), gA

    def adjoint_sensitivity(self, g, u, tol=1e-12, maxit=2000, precond="mg") -> dict:
        """For the step assembled last and its solution u: lambda = K^-1 g and per property set the
        derivatives through u with respect to log stiffness (dlogE) and log thermal strain (dlogA)."""
        g = np.ascontiguousarray(g, np.float64); u = np.ascontiguousarray(u, np.float64)
        dE = np.zeros(self.pkg.npset); dA = np.zeros(self.pkg.npset)
        info = TmSolveInfo()
        o = self.make_opts(tol, maxit, 0, precond, "fp64", -1)
        vp = lambda a: a.ctypes.data_as(C.c_void_p)
        check(load().tm_adjoint_sensitivity(self.h, vp(g), vp(u), C.byref(o), vp(dE), vp(dA), C.byref(info)), allow_not_converged=True)
        return dict(dlogE=dE, dlogA=dA, adjoint=self.record(info, "adjoint", precond))

    def set_sublayers(self, step: StepData):
        """The step's sub-layers of the layered property sets, for the stress histories (call
        after prepare_step / assemble_step of that step)."""
        vp = lambda a: a.ctypes.data_as(C.c_void_p)
        n = np.ascontiguousarray(step.sub_n if step.sub_n is not None else np.zeros(len(step.layered)), np.int32)
        z = np.ascontiguousarray(step.sub_z if step.sub_z is not None and len(step.sub_z) else np.zeros(2), np.float64)
        d = np.ascontiguousarray(step.sub_D if step.sub_D is not None and len(step.sub_D) else np.zeros(36), np.float64)
        s0 = np.ascontiguousarray(step.sub_s0 if step.sub_s0 is not None and len(step.sub_s0) else np.zeros(6), np.float64)
        check(load().tm_set_sublayers(self.h, vp(n), vp(z), vp(d), vp(s0)))

    def accumulate_state(self, du, elems, stride: int, state: np.ndarray) -> np.ndarray:
        """Model.accumulateStep (src/core/09-assembly.js:508-544): state (nel x stride, updated in
        place) += q's increment and the sub-layer stress monomials of the step loaded last."""
        du = np.ascontiguousarray(du, np.float64); elems = np.ascontiguousarray(elems, np.int32)
        if state.dtype != np.float64 or not state.flags.c_contiguous or state.size != stride * len(elems):
            raise ValueError("state must be a contiguous float64 array of stride values per element")
        vp = lambda a: a.ctypes.data_as(C.c_void_p)
        check(load().tm_accumulate_state(self.h, vp(du), len(elems), vp(elems), int(stride), vp(state)))
        return state

    def state_stress(self, elem, state, stride: int, nat) -> tuple:
        """stateStress (src/core/09-assembly.js:555-571): (eps, sig), (npts, 6) each."""
        elem = np.ascontiguousarray(elem, np.int32)
        state = np.ascontiguousarray(state, np.float64).reshape(-1); nat = np.ascontiguousarray(nat, np.float64).reshape(-1)
        if state.size != stride * len(elem) or nat.size != 3 * len(elem):
            raise ValueError("state needs stride and nat 3 values per point")
        eps = np.zeros(6 * len(elem)); sig = np.zeros(6 * len(elem))
        vp = lambda a: a.ctypes.data_as(C.c_void_p)
        check(load().tm_state_stress(self.h, len(elem), vp(elem), vp(state), int(stride), vp(nat), vp(eps), vp(sig)))
        return eps.reshape(-1, 6), sig.reshape(-1, 6)

    def sample_plane(self, u, k: int, comp: int, x, y) -> np.ndarray:
        """samplePlane (src/core/12-post.js:30-38) of the nodal field u at the points (x, y)."""
        u = np.ascontiguousarray(u, np.float64)
        x = np.ascontiguousarray(x, np.float64).reshape(-1); y = np.ascontiguousarray(y, np.float64).reshape(-1)
        if u.size != self.ndof or x.size != y.size:
            raise ValueError("u must hold one value per DOF and x, y one per point")
        out = np.zeros(len(x))
        check(load().tm_sample_plane(self.h, u.ctypes.data_as(C.c_void_p), int(k), int(comp), len(x),
                                     x.ctypes.data_as(C.c_void_p), y.ctypes.data_as(C.c_void_p),
                                     out.ctypes.data_as(C.c_void_p)))
        return out

    # ---- LinearSolver.solve ----------------------------------------------------------------
    @staticmethod
    def make_opts(tol=1e-8, maxit=2000, warm=20, precond="mg", precision="fp64", key=-1) -> TmSolveOpts:
        o = TmSolveOpts()
        load().tm_default_solve_opts(C.byref(o))
        o.tol = tol; o.maxit = maxit; o.warm = warm
        o.precond = _lib.PRECONDS[precond]
        o.precision = {"fp64": 0, "mixed": 1, "mixed_ir": 2}[precision]
        o.key = -1 if key is None else int(key)
        return o

    @staticmethod
    def record(info: TmSolveInfo, label=None, precond="mg") -> dict:
        fb = None
        if info.fallback:
            fb = dict(first=_lib.PRECOND_NAMES.get(int(info.fallback_first), "?"), iters=int(info.fallback_iters),
                      relres=float(info.fallback_relres))
        return dict(label=label, iters=int(info.iters), relres=float(info.relres), converged=bool(info.converged),
                    ms=float(info.ms), pcMs=float(info.pc_ms), precond=_lib.PRECOND_NAMES.get(int(info.precond), precond),
                    rebuilt=bool(info.rebuilt), warm=int(info.warm), iters0=float(info.iters0), fallback=fb,
                    jitter=int(info.jitter_count), levels=int(info.levels), refinements=int(info.refinements))

    def pc_apply(self, r) -> np.ndarray:
        """z = M^-1 r with the preconditioner the last solve built (scaled space; pc.apply)."""
        r = np.ascontiguousarray(r, np.float64)
        z = np.zeros(self.ndof)
        check(load().tm_pc_apply(self.h, r.ctypes.data_as(C.c_void_p), z.ctypes.data_as(C.c_void_p)))
        return z

    def vcycle_shapes(self) -> dict:
        """Launch shapes the FP32 V-cycle's autotuner chose: warps per block of the shell sweep and
        residual per tuned level, and the TMA level-0 sweep's stage count (0: not used)."""
        cap = 32
        n, st = C.c_int32(0), C.c_int32(0)
        ws, wa = (C.c_int32 * cap)(), (C.c_int32 * cap)()
        check(load().tm_vcycle_shapes(self.h, cap, C.byref(n), ws, wa, C.byref(st)))
        k = min(n.value, cap)
        return dict(wpb_sweep=list(ws[:k]), wpb_apply=list(wa[:k]), tma_stages=st.value)

    def set_wait_test(self, on: bool):
        """Test hook of the timeout path: the level-0 TMA sweep waits for a flag that nothing sets."""
        check(load().tm_set_wait_test(self.h, 1 if on else 0))

    def clear_warm(self):
        """Drops the warm start's stored solutions (tm_clear_warm)."""
        check(load().tm_clear_warm(self.h))

    def set_level0(self, matrix_free: bool):
        """Level-0 operator of the solves after the next assembly: the assembled stencil (default)
        or cell-by-cell products with the element classes' matrices (tm_set_level0)."""
        check(load().tm_set_level0(self.h, 1 if matrix_free else 0))

    @property
    def level0_matrix_free(self) -> bool:
        """Whether the current step's level-0 operator is the matrix-free one."""
        v = C.c_int32(0)
        check(load().tm_level0(self.h, C.byref(v)))
        return bool(v.value)

    def mg_levels(self) -> list:
        """The multigrid hierarchy, fine to coarse: (nx, ny, nn, b) per level (MultigridPC's levels)."""
        cap = 64
        n = C.c_int32(0)
        out = np.zeros(4 * cap, np.int32)
        check(load().tm_mg_levels(self.h, cap, out.ctypes.data_as(C.c_void_p), C.byref(n)))
        return [tuple(int(v) for v in out[4 * l:4 * l + 4]) for l in range(min(n.value, cap))]

    def shell_sweep_bytes(self):
        """(algorithmic bytes, launches) of the shell-level column sweeps of one FP32 V-cycle."""
        b = C.c_double(); n = C.c_int32()
        check(load().tm_shell_sweep_bytes(self.h, C.byref(b), C.byref(n)))
        return float(b.value), int(n.value)

    def mg_node_agg(self) -> np.ndarray:
        """Level-1 aggregate of every node (buildShellLevel's grouping)."""
        out = np.zeros(self.nn, np.int32)
        check(load().tm_mg_node_agg(self.h, out.ctypes.data_as(C.c_void_p)))
        return out

    def set_vcycle_shapes(self, wpb_sweep=None, wpb_apply=None, tma_stages=0):
        """Pin the FP32 V-cycle's launch shapes (as vcycle_shapes returns them); None: autotune."""
        if wpb_sweep is None:
            check(load().tm_set_vcycle_shapes(self.h, -1, None, None, 0))
            return
        n = len(wpb_sweep)
        ws, wa = (C.c_int32 * max(n, 1))(*wpb_sweep), (C.c_int32 * max(n, 1))(*wpb_apply)
        check(load().tm_set_vcycle_shapes(self.h, n, ws, wa, int(tma_stages)))

    def solve(self, f, label=None, key=-1, tol=1e-8, maxit=2000, warm=20, precond="mg", precision="fp64",
              out: Optional[np.ndarray] = None, progress=None, progress_every: int = 1) -> dict:
        """LinearSolver.solve with host arrays; the displacement goes to `out` when given.
        progress(it, relres), when given, is called between PCG iterations every progress_every
        iterations, on this thread (the reference's LIVE.post progress, 10-solver.js:1033)."""
        f = np.ascontiguousarray(f, np.float64)
        u = _out_array(out, self.ndof)
        info = TmSolveInfo()
        o = self.make_opts(tol, maxit, warm, precond, precision, key)
        if progress is not None:
            cb = _lib.PROGRESS_FN(lambda user, it, rel: progress(int(it), float(rel)))
            o.progress = cb
            o.progress_every = int(progress_every)
        check(load().tm_solve(self.h, f.ctypes.data_as(C.c_void_p), u.ctypes.data_as(C.c_void_p), C.byref(o), C.byref(info)),
              allow_not_converged=True)
        rec = self.record(info, label, precond)
        self.log.append(rec)
        rec = dict(rec)
        rec["u"] = u
        return rec

    def solve_f32(self, f, label=None, key=-1, tol=1e-8, maxit=2000, warm=20, precond="mg", precision="fp64") -> dict:
        """solve with the displacement returned as float32 (the increment the analysis keeps)."""
        f = np.ascontiguousarray(f, np.float64)
        u = np.zeros(self.ndof, np.float32)
        info = TmSolveInfo()
        o = self.make_opts(tol, maxit, warm, precond, precision, key)
        check(load().tm_solve_f32(self.h, f.ctypes.data_as(C.c_void_p), u.ctypes.data_as(C.c_void_p), C.byref(o), C.byref(info)),
              allow_not_converged=True)
        rec = self.record(info, label, precond)
        self.log.append(rec)
        rec = dict(rec)
        rec["u"] = u
        return rec

    def warpage_sensitivity(self, u, k: int = 0, tol=1e-12, maxit=2000, precond="mg") -> dict:
        """Adjoint sensitivities of J = mean squared residual of plane k's z displacements about
        their least-squares plane, for the solution u of the step assembled last: J and, per
        property set, dJ/dlog(E) and dJ/dlog(alpha) (tm_warpage_sensitivity)."""
        u = np.ascontiguousarray(u, np.float64)
        J = C.c_double()
        dE = np.zeros(self.pkg.npset); dA = np.zeros(self.pkg.npset)
        info = TmSolveInfo()
        o = self.make_opts(tol, maxit, 0, precond, "fp64", -1)
        vp = lambda a: a.ctypes.data_as(C.c_void_p)
        check(load().tm_warpage_sensitivity(self.h, vp(u), int(k), C.byref(o), C.byref(J), vp(dE), vp(dA), C.byref(info)),
              allow_not_converged=True)
        return dict(J=J.value, dlogE=dE, dlogA=dA, adjoint=self.record(info, "adjoint", precond))

    def sensitivity_direction(self, base: StepData, direction: StepData) -> np.ndarray:
        """After warpage_sensitivity: dJ/dt per property set for the parameter whose derivative of
        the set data (D, s0 or W, V) is `direction` (tm_sensitivity_direction)."""
        sb, kb = self._step_struct(base)
        sd, kd = self._step_struct(direction)
        out = np.zeros(self.pkg.npset)
        check(load().tm_sensitivity_direction(self.h, C.byref(sb), C.byref(sd), out.ctypes.data_as(C.c_void_p)))
        return out

    def solve_device(self, f_ptr: int, u_ptr: int, tol=1e-8, maxit=2000, warm=20, precond="mg", precision="fp64", key=-1) -> dict:
        """The same solve with f and u already in device memory (raw device pointers)."""
        info = TmSolveInfo()
        o = self.make_opts(tol, maxit, warm, precond, precision, key)
        check(load().tm_solve_device(self.h, C.c_void_p(f_ptr), C.c_void_p(u_ptr), C.byref(o), C.byref(info)),
              allow_not_converged=True)
        return self.record(info, None, precond)


    # ---- stream and measurement hooks ----------------------------------------------------------
    def set_stream(self, stream_ptr: int):
        """Run on the caller's CUDA stream (e.g. torch.cuda.current_stream().cuda_stream)."""
        check(load().tm_set_stream(self.h, C.c_void_p(stream_ptr)))

    def time_kernel(self, name: Optional[str]):
        """Bracket every launch of one kernel class with CUDA events (None: off)."""
        check(load().tm_kernel_timer(self.h, -1 if name is None else _lib.KERNELS[name]))

    def kernel_time(self):
        """(launches, summed device ms) of the timed kernel class since time_kernel()."""
        n = C.c_int64(); ms = C.c_double()
        check(load().tm_kernel_timer_read(self.h, C.byref(n), C.byref(ms)))
        return int(n.value), float(ms.value)


def launch_count() -> int:
    """Kernels launched by libtmsolve.so since it was loaded."""
    return int(load().tm_launch_count())


__all__ = ["DeviceModel", "TmError", "launch_count"]


def device_peaks() -> dict:
    """CUDA-core FMA throughput of the current device (TFLOP/s, FP32 and FP64)."""
    f32, f64 = C.c_double(), C.c_double()
    check(load().tm_device_peaks(C.byref(f32), C.byref(f64)))
    return dict(fp32_tflops=f32.value, fp64_tflops=f64.value)
