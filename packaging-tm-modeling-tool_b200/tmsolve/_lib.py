"""ctypes binding of libtmsolve.so (C-ABI declared in include/tmsolve.h).

The library is required: there is no CPU fallback. Loading fails loudly when the
built shared object is missing.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
PKG_ROOT = os.path.dirname(HERE)
LIB_PATH = os.path.join(PKG_ROOT, "lib", "libtmsolve.so")

TM_OK, TM_NOT_CONVERGED, TM_NONFINITE, TM_TIMEOUT, TM_BAD_INPUT, TM_CUDA, TM_NO_DEVICE = range(7)
STATUS_NAMES = {0: "TM_OK", 1: "TM_NOT_CONVERGED", 2: "TM_NONFINITE", 3: "TM_TIMEOUT", 4: "TM_BAD_INPUT", 5: "TM_CUDA",
                6: "TM_NO_DEVICE"}

EXPORTED = ["tm_default_solve_opts", "tm_create", "tm_assemble_step", "tm_set_bcsr", "tm_solve", "tm_matvec", "tm_get_bcsr",
            "tm_sizes", "tm_destroy", "tm_last_error", "tm_solve_device", "tm_matvec_device", "tm_anand_screen",
            "tm_anand_screen_device", "tm_anand_step", "tm_set_stream", "tm_launch_count", "tm_kernel_timer",
            "tm_kernel_timer_read", "tm_assemble_step_device", "tm_prepare_step", "tm_accumulate_q", "tm_accumulate_q_device",
            "tm_element_strains", "tm_element_strains_device", "tm_sample_plane", "tm_sample_plane_device",
            "tm_anand_screen_pillar", "tm_anand_screen_pillar_device", "tm_pc_apply", "tm_pc_apply_device",
            "tm_submodel_create", "tm_submodel_destroy", "tm_submodel_sizes", "tm_submodel_step", "tm_submodel_get",
            "tm_submodel_run", "tm_submodel_run_batch", "tm_set_sublayers", "tm_accumulate_state",
            "tm_accumulate_state_device", "tm_state_stress", "tm_state_stress_device", "tm_solve_f32",
            "tm_warpage_sensitivity", "tm_sensitivity_direction", "tm_vcycle_shapes", "tm_set_vcycle_shapes", "tm_submodel_run_sections", "tm_submodel_stress_snapshot",
            "tm_mg_levels", "tm_mg_node_agg", "tm_shell_sweep_bytes", "tm_device_peaks",
            "tm_set_wait_test", "tm_anand_screen_gradient",
            "tm_element_strains_adjoint", "tm_accumulate_q_adjoint", "tm_adjoint_sensitivity", "tm_set_level0", "tm_level0", "tm_clear_warm", "tm_submodel_set_precond", "tm_submodel_counters"]
PRECONDS = {"mg": 0, "jacobi": 1, "ic": 2}
PRECOND_NAMES = {v: k for k, v in PRECONDS.items()}
KERNELS = dict(apply0=0, sweep_solid=1, sweep_shell=2, assemble=3, galerkin01=4, apply_shell=5, setup_level0=6, setup_shell=7,
               setup_coarsest=8, to_fp32=9)

dp = C.POINTER(C.c_double)
ip = C.POINTER(C.c_int32)


class TmMesh(C.Structure):
    _fields_ = [("nx", C.c_int32), ("ny", C.c_int32), ("nz", C.c_int32),
                ("xs", dp), ("ys", dp), ("zs", dp), ("nn", C.c_int32), ("ne", C.c_int32),
                ("coords", dp), ("nodeId", ip), ("conn", ip), ("eIJK", ip), ("colStart", ip), ("cellElems", ip),
                ("eGroup", ip), ("ePart", C.POINTER(C.c_int8)), ("eScale", dp), ("ngroups", C.c_int32), ("groupStage", ip),
                ("npset", C.c_int32), ("ePset", ip), ("nconstr", C.c_int32), ("constr", ip),
                ("nfeatureX", C.c_int32), ("nfeatureY", C.c_int32), ("featureX", ip), ("featureY", ip),
                ("nmodconstr", C.c_int32), ("modconstr", ip)]


class TmStep(C.Structure):
    _fields_ = [("stage", C.c_int32), ("psetLayered", ip), ("D", dp), ("s0", dp), ("W", dp), ("V", dp), ("psetBorn", ip)]


PROGRESS_FN = C.CFUNCTYPE(None, C.c_void_p, C.c_int32, C.c_double)


class TmSolveOpts(C.Structure):
    _fields_ = [("tol", C.c_double), ("maxit", C.c_int32), ("warm", C.c_int32), ("precond", C.c_int32),
                ("precision", C.c_int32), ("key", C.c_int64), ("progress", PROGRESS_FN), ("progress_user", C.c_void_p),
                ("progress_every", C.c_int32)]


class TmSolveInfo(C.Structure):
    _fields_ = [("iters", C.c_int32), ("relres", C.c_double), ("iters0", C.c_double), ("converged", C.c_int32),
                ("ms", C.c_double), ("pc_ms", C.c_double), ("rebuilt", C.c_int32), ("warm", C.c_int32),
                ("fallback", C.c_int32), ("jitter_count", C.c_int32), ("levels", C.c_int32), ("status", C.c_int32),
                ("refinements", C.c_int32), ("precond", C.c_int32), ("fallback_first", C.c_int32),
                ("fallback_iters", C.c_int32), ("fallback_relres", C.c_double)]


class TmAnandMaterial(C.Structure):
    _fields_ = [("A", C.c_double), ("QR", C.c_double), ("xi", C.c_double), ("m", C.c_double), ("shat", C.c_double),
                ("n", C.c_double), ("h0", C.c_double), ("a", C.c_double), ("s0", C.c_double), ("nu", C.c_double),
                ("Etab", dp), ("Ftab", dp)]


class TmPillar(C.Structure):
    _fields_ = [("fs", C.c_double), ("nu", C.c_double), ("Etab", dp), ("Ftab", dp)]


class TmSubmodelSpec(C.Structure):
    _fields_ = [("nx", C.c_int32), ("ny", C.c_int32), ("nz", C.c_int32), ("xs", dp), ("ys", dp), ("zs", dp), ("cellMat", ip),
                ("nglob", C.c_int32), ("nt", C.c_int32), ("ts", dp), ("fields", dp), ("u25", dp), ("nb", C.c_int32),
                ("bGlob", ip), ("bW", dp), ("solder", TmAnandMaterial), ("elasticSolder", C.c_int32), ("ufE", dp), ("ufF", dp),
                ("ufNu", C.c_double), ("siD", dp), ("siF", dp), ("subD", dp), ("subF", dp), ("nuMax", C.c_double),
                ("zt", C.c_double), ("zaf", C.c_double), ("uniformMaterial", C.c_int32), ("density", C.c_double),
                ("nuMaxGlobal", C.c_double), ("nsec", C.c_int32), ("secZ", dp), ("secD", dp), ("secF", dp)]


_lib = None


def load():
    """Load libtmsolve.so; raises when it has not been built (there is no CPU fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"libtmsolve.so not found at {LIB_PATH}: build it with `make -C {PKG_ROOT}` "
                          "(the solve path has no CPU fallback)")
    L = C.CDLL(LIB_PATH)
    vp = C.c_void_p
    L.tm_default_solve_opts.argtypes = [C.POINTER(TmSolveOpts)]
    L.tm_create.argtypes = [C.POINTER(TmMesh), C.POINTER(vp)]
    L.tm_assemble_step.argtypes = [vp, C.POINTER(TmStep), vp]
    L.tm_assemble_step_device.argtypes = [vp, C.POINTER(TmStep), vp]
    L.tm_set_bcsr.argtypes = [vp, vp, vp, vp, vp]
    L.tm_solve.argtypes = [vp, vp, vp, C.POINTER(TmSolveOpts), C.POINTER(TmSolveInfo)]
    L.tm_solve_device.argtypes = [vp, vp, vp, C.POINTER(TmSolveOpts), C.POINTER(TmSolveInfo)]
    L.tm_solve_f32.argtypes = [vp, vp, vp, C.POINTER(TmSolveOpts), C.POINTER(TmSolveInfo)]
    L.tm_sensitivity_direction.argtypes = [vp, C.POINTER(TmStep), C.POINTER(TmStep), vp]
    L.tm_warpage_sensitivity.argtypes = [vp, vp, C.c_int32, C.POINTER(TmSolveOpts), vp, vp, vp, C.POINTER(TmSolveInfo)]
    L.tm_matvec.argtypes = [vp, vp, vp]
    L.tm_matvec_device.argtypes = [vp, vp, vp]
    L.tm_pc_apply.argtypes = [vp, vp, vp]
    L.tm_submodel_create.argtypes = [C.POINTER(TmSubmodelSpec), C.POINTER(vp)]
    L.tm_submodel_destroy.argtypes = [vp]
    L.tm_submodel_set_precond.argtypes = [vp, C.c_int32]
    L.tm_submodel_counters.argtypes = [vp, vp]
    L.tm_submodel_sizes.argtypes = [vp, vp]
    L.tm_submodel_step.argtypes = [vp, C.c_double, C.c_double, vp, vp, vp]
    L.tm_submodel_get.argtypes = [vp, vp, vp, vp]
    L.tm_submodel_run.argtypes = [vp, C.c_int32, vp, vp, vp, C.c_int32, C.c_double, C.c_double, vp, vp, vp]
    L.tm_submodel_run_sections.argtypes = [vp, C.c_int32, vp, vp, vp, vp, C.c_int32, C.c_double, C.c_double, vp, vp, vp, C.c_int32,
                                           vp, vp, vp]
    L.tm_submodel_stress_snapshot.argtypes = [vp, C.c_double, vp]
    L.tm_submodel_run_batch.argtypes = [C.c_int32, vp, C.c_int32, vp, vp, vp, C.c_int32, vp, vp, vp, vp, vp, vp]
    L.tm_pc_apply_device.argtypes = [vp, vp, vp]
    L.tm_vcycle_shapes.argtypes = [vp, C.c_int32, vp, vp, vp, vp]
    L.tm_set_vcycle_shapes.argtypes = [vp, C.c_int32, vp, vp, C.c_int32]
    L.tm_mg_levels.argtypes = [vp, C.c_int32, vp, vp]
    L.tm_shell_sweep_bytes.argtypes = [vp, vp, vp]
    L.tm_mg_node_agg.argtypes = [vp, vp]
    L.tm_device_peaks.argtypes = [vp, vp]
    L.tm_set_wait_test.argtypes = [vp, C.c_int32]
    L.tm_set_level0.argtypes = [vp, C.c_int32]
    L.tm_level0.argtypes = [vp, vp]
    L.tm_clear_warm.argtypes = [vp]
    L.tm_element_strains_adjoint.argtypes = [vp, C.c_int32, vp, vp, vp, vp]
    L.tm_accumulate_q_adjoint.argtypes = [vp, C.c_int32, vp, vp, vp, vp]
    L.tm_adjoint_sensitivity.argtypes = [vp, vp, vp, C.POINTER(TmSolveOpts), vp, vp, C.POINTER(TmSolveInfo)]
    L.tm_anand_screen_gradient.argtypes = [vp, vp, C.c_int32, vp, vp, C.c_int32, vp, vp, vp, vp, C.c_int32] + [vp] * 4
    L.tm_get_bcsr.argtypes = [vp, vp, vp, vp]
    L.tm_sizes.argtypes = [vp, C.POINTER(C.c_int64)]
    L.tm_destroy.argtypes = [vp]
    L.tm_last_error.argtypes = [C.c_char_p, C.c_size_t]
    L.tm_last_error.restype = C.c_int32
    L.tm_anand_screen.argtypes = [C.POINTER(TmAnandMaterial), C.c_int32, C.c_int32, vp, vp, C.c_int32, vp, vp, vp, vp,
                                  C.c_int32, vp, vp, vp]
    L.tm_anand_screen_device.argtypes = L.tm_anand_screen.argtypes
    L.tm_anand_screen_pillar.argtypes = [C.POINTER(TmAnandMaterial), C.POINTER(TmPillar)] + L.tm_anand_screen.argtypes[1:]
    L.tm_anand_screen_pillar_device.argtypes = L.tm_anand_screen_pillar.argtypes
    L.tm_anand_screen_noalloc.argtypes = L.tm_anand_screen.argtypes + [vp]
    L.tm_anand_screen_noalloc.restype = C.c_int32
    L.tm_anand_step.argtypes = [C.POINTER(TmAnandMaterial), C.c_int32, vp, vp, C.c_double, C.c_double, vp, vp, C.c_int32]
    L.tm_set_stream.argtypes = [vp, vp]
    L.tm_launch_count.argtypes = []
    L.tm_kernel_timer.argtypes = [vp, C.c_int32]
    L.tm_kernel_timer_read.argtypes = [vp, C.POINTER(C.c_int64), C.POINTER(C.c_double)]
    L.tm_prepare_step.argtypes = [vp, C.POINTER(TmStep)]
    L.tm_set_sublayers.argtypes = [vp, vp, vp, vp, vp]
    L.tm_accumulate_state.argtypes = [vp, vp, C.c_int32, vp, C.c_int32, vp]
    L.tm_accumulate_state_device.argtypes = L.tm_accumulate_state.argtypes
    L.tm_state_stress.argtypes = [vp, C.c_int32, vp, vp, C.c_int32, vp, vp, vp]
    L.tm_state_stress_device.argtypes = L.tm_state_stress.argtypes
    L.tm_accumulate_q.argtypes = [vp, vp, C.c_int32, vp, vp]
    L.tm_accumulate_q_device.argtypes = L.tm_accumulate_q.argtypes
    L.tm_element_strains.argtypes = [vp, C.c_int32, vp, vp, vp, vp]
    L.tm_element_strains_device.argtypes = L.tm_element_strains.argtypes
    L.tm_sample_plane.argtypes = [vp, vp, C.c_int32, C.c_int32, C.c_int32, vp, vp, vp]
    L.tm_sample_plane_device.argtypes = L.tm_sample_plane.argtypes
    for name in EXPORTED:
        getattr(L, name).restype = C.c_int32 if name not in ("tm_default_solve_opts",) else None
    L.tm_launch_count.restype = C.c_int64
    _lib = L
    return L


class TmError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {msg}")
        self.status = status


def last_error() -> str:
    L = load()
    buf = C.create_string_buffer(4096)
    L.tm_last_error(buf, 4096)
    return buf.value.decode(errors="replace")


def check(status: int, allow_not_converged: bool = False) -> int:
    if status == TM_OK or (allow_not_converged and status == TM_NOT_CONVERGED):
        return status
    raise TmError(status, last_error())
