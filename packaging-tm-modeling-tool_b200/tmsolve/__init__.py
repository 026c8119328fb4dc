"""tmsolve: B200 solve path of the FCBGA thermomechanical tool (host side).

The GPU library (``libtmsolve.so``, C-ABI in ``include/tmsolve.h``) holds the
stiffness assembly and apply, the PCG solver with the semi-coarsening multigrid
preconditioner and the Anand return map. This package is the host-side mirror
of the reference's solver interface (``LinearSolver``, src/core/10-solver.js)
over that C-ABI, plus the synthetic package inputs used by the tests and the
benchmark.
"""
from .mesh import Mesh, build_structured_mesh, constraints321  # noqa: F401
from .packages import Package, StepData, box_package, fcbga_c1, lidded_c2  # noqa: F401
