/*
 * tmsolve.h -- C-ABI of the B200 solve path of the FCBGA thermomechanical tool.
 *
 * The reference tool (ProtonNeutronElectron69/Packaging-TM-modeling-tool) is
 * JavaScript; its solve path runs inside the compute worker's driver thread.
 * This library replaces, behind a thin context-aware N-API addon, the
 * following reference interfaces (paths relative to the reference project):
 *
 *   tm_create          new FEModel(mesh, cfg) + new LinearSolver(model, opts)
 *                      src/core/09-assembly.js:208-233, src/core/10-solver.js:826-841
 *   tm_assemble_step   FEModel.assembleStep(Ta, Tb, stage, rhs) with applyConstraints
 *                      src/core/09-assembly.js:392-424, 445-464 (prepareStep's per-group
 *                      data, :346-365, is computed by the caller and passed in tm_step)
 *   tm_set_bcsr        the assembled model.pattern / model.val / model.isConstrained that
 *                      LinearSolver reads (src/core/09-assembly.js:220-223, 445-450)
 *   tm_solve           LinearSolver.solve(f, label, key)  src/core/10-solver.js:933-994
 *   tm_matvec          fullMatVec(P, val, x, y)           src/core/09-assembly.js:151-165
 *   tm_anand_screen    screenJoints' per-site Anand loop  src/core/13-fatigue.js:395-451
 *                      (AnandPoint.stepColumn / step, :13-166)
 *   tm_anand_screen_pillar  screenDdi's joints: solder caps on elastic pillars
 *                      (AnandPoint.stepSeriesColumn, src/core/13-fatigue.js:178-206, 369-376, 404-433)
 *   tm_anand_step      AnandPoint.step + commit           src/core/13-fatigue.js:67-143, 229-232
 *   tm_prepare_step    FEModel.stepRecovery(Ta, Tb, stage): the step's shape matrices and element
 *                      thermal loads without an assembly (src/core/09-assembly.js:480-491)
 *   tm_accumulate_q    Model.accumulateStep(e, rec, du, state, qOnly = true) over a list of
 *                      elements (src/core/09-assembly.js:508-533, with stepRecovery :480-491),
 *                      the march of Analysis.qAlong (src/core/11-analysis.js:298-316)
 *   tm_element_strains boxStrainAt at natural points (src/core/07-element.js:127-142), the
 *                      inner loop of siteStrainTable (src/core/13-fatigue.js:318-346)
 *   tm_accumulate_state / tm_state_stress  Model.accumulateStep and stateStress
 *                      (src/core/09-assembly.js:508-571), the element histories of StateView.point
 *                      (src/core/11-analysis.js:343-379) behind dieSurfaceStress and jointLoads
 *   tm_submodel_*      BumpSubmodel (src/core/13-fatigue.js:470-1104): create, stepTo, run
 *   tm_sample_plane    samplePlane(mesh, u, k, comp, x, y) at many points
 *                      (src/core/12-post.js:30-38), the sampler of warpageJEITA (:60-109)
 *
 * Conventions
 *   - Node, element and DOF numbering are the mesher's, taken verbatim
 *     (src/core/06-mesher.js:14-72): nodes z fastest then y then x, DOF = 3*node + comp.
 *   - Host buffers passed in are read during the call and never retained; the
 *     context owns all device memory. Output buffers are caller-allocated.
 *   - Every entry point returns a tm_status; TM_NOT_CONVERGED is the only
 *     non-error status (the addon maps it to converged:false, everything else to
 *     a thrown Error, as LinearSolver's callers expect: src/core/11-analysis.js:204).
 *   - One context per calling thread; calls are synchronous on that thread.
 *   - There is no CPU fallback: without a usable sm_100 GPU, tm_create returns TM_NO_DEVICE.
 */
#ifndef TMSOLVE_H
#define TMSOLVE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int tm_status;
#define TM_OK 0
#define TM_NOT_CONVERGED 1   /* PCG did not reach tol (converged:false in the reference record) */
#define TM_NONFINITE 2       /* NaN/Inf in the input or during the iteration */
#define TM_TIMEOUT 3         /* a bounded device wait ran out */
#define TM_BAD_INPUT 4       /* inconsistent sizes, indices or call order */
#define TM_CUDA 5            /* a CUDA runtime error */
#define TM_NO_DEVICE 6       /* no sm_100 device available: there is no CPU fallback */

typedef struct tm_ctx tm_ctx;

/* The mesher's output (buildStructuredMesh, 06-mesher.js:66-71) plus the element
 * property-set map and the constraint DOFs (constraints321, 06-mesher.js:112-116). */
typedef struct {
  int32_t nx, ny, nz;            /* grid lines in x, y and z planes */
  const double* xs;              /* nx */
  const double* ys;              /* ny */
  const double* zs;              /* nz */
  int32_t nn, ne;                /* nodes, elements */
  const double* coords;          /* 3*nn */
  const int32_t* nodeId;         /* nx*ny*nz, -1 where no node */
  const int32_t* conn;           /* 8*ne, local order loc of 06-mesher.js:49 */
  const int32_t* eIJK;           /* 3*ne */
  const int32_t* colStart;       /* nx*ny+1 */
  const int32_t* cellElems;      /* 2*(nx-1)*(ny-1)*(nz-1), -1 where no phase */
  const int32_t* eGroup;         /* ne */
  const int8_t* ePart;           /* ne, PART ids of 06-mesher.js:3-4 */
  const double* eScale;          /* ne */
  int32_t ngroups;
  const int32_t* groupStage;     /* ngroups: birth stage of every group (09-assembly.js:339) */
  int32_t npset;                 /* property sets: homogeneous groups and layered sections */
  const int32_t* ePset;          /* ne: property set of every element (group, or section of its layer) */
  int32_t nconstr;
  const int32_t* constr;         /* constrained DOFs */
  int32_t nfeatureX, nfeatureY;  /* feature lines kept at every multigrid level (06-mesher.js:504) */
  const int32_t* featureX;
  const int32_t* featureY;
  int32_t nmodconstr;            /* stacked modules: each module's 3-2-1 support DOFs (mesh.moduleConstraints,
                                    06-mesher.js:535-545); 0 for a package without modules */
  const int32_t* modconstr;
} tm_mesh;

/* Stacked-module stages (stage < 0 on a mesh with module supports, 09-assembly.js:392-443): only the
 * elements born in the stage are assembled, the constrained DOFs are the package's and every module's
 * 3-2-1 supports plus all DOFs of the nodes no born element touches, and the multigrid hierarchy is
 * built over the born elements and the nodes they touch (10-solver.js:260-266); the first solve after
 * the active set changes builds that hierarchy. */
/* Per-step property sets (FEModel.prepareStep's output, 09-assembly.js:346-365):
 * homogeneous: mean stiffness D (36) and thermal stress increment s0 (6);
 * layered: step-mean weights W_j (3 x 36) and thermal weights V_j (3 x 6). */
typedef struct {
  int32_t stage;                 /* element birth: group stage <= stage (09-assembly.js:401-403) */
  const int32_t* psetLayered;    /* npset, 0 or 1 */
  const double* D;               /* 36*npset (homogeneous sets) */
  const double* s0;              /* 6*npset */
  const double* W;               /* 108*npset (layered sets) */
  const double* V;               /* 18*npset */
  const int32_t* psetBorn;       /* npset: thermal load of the set on (sec._born / g._born) */
} tm_step;

#define TM_PC_MG 0
#define TM_PC_JACOBI 1       /* diagonal scaling only (no counterpart in the reference; a baseline) */
#define TM_PC_IC 2           /* IC(0) with Manteuffel shift (ICPC, src/core/10-solver.js:741-800) */
#define TM_PREC_FP64 0       /* everything in FP64 */
#define TM_PREC_MIXED 1      /* FP64 PCG (apply, residuals, dots); the whole V-cycle in FP32 except the FP64 coarsest solve */
#define TM_PREC_MIXED_IR 2   /* FP64 iterative refinement of an FP32 MG-PCG (FP32 apply and V-cycle); on a sweep that
                                fails to halve the FP64 residual it continues as TM_PREC_MIXED */

typedef struct {
  double tol;                    /* relative residual in the scaled 2-norm (PCG_TOL 1e-8) */
  int32_t maxit;                 /* PCG_MAXIT 2000 */
  int32_t warm;                  /* stored solutions for the warm start (WARM_START_MAX 20), 0 = off */
  int32_t precond;               /* preferred kind: TM_PC_MG, TM_PC_IC or TM_PC_JACOBI; a run that fails after a
                                    rebuild falls back once to the other kind (MG <-> IC, 10-solver.js:967-976) */
  int32_t precision;             /* TM_PREC_FP64, TM_PREC_MIXED or TM_PREC_MIXED_IR */
  int64_t key;                   /* preconditioner key (solve(f, label, key)); -1 = none */
  void (*progress)(void* user, int32_t it, double relres);  /* called between iterations, may be NULL */
  void* progress_user;
  int32_t progress_every;        /* iterations between progress calls */
} tm_solve_opts;

typedef struct {
  int32_t iters;                 /* total PCG iterations of the solve (res.iters) */
  double relres;                 /* final relative residual */
  double iters0;                 /* relative residual of the initial guess (res.iters0) */
  int32_t converged;
  double ms;                     /* wall time of the solve */
  double pc_ms;                  /* preconditioner set-up time */
  int32_t rebuilt;               /* a preconditioner was (re)built in this solve */
  int32_t warm;                  /* stored solutions after the solve */
  int32_t fallback;              /* fell back to another preconditioner */
  int32_t jitter_count;          /* jittered pivots of the column factors (10-solver.js:61-64, 490) */
  int32_t levels;                /* multigrid levels */
  int32_t status;
  int32_t refinements;           /* mixed precision: outer FP64 refinement sweeps */
  int32_t precond;               /* kind of the preconditioner the solve ended with (rec.precond) */
  int32_t fallback_first;        /* with fallback: the kind that failed, its iterations and residual */
  int32_t fallback_iters;
  double fallback_relres;
} tm_solve_info;

/* Library defaults for tm_solve_opts (the reference's CONST values). */
void tm_default_solve_opts(tm_solve_opts* opts);

/* Creates the device model of a mesh (FEModel + LinearSolver). */
tm_status tm_create(const tm_mesh* mesh, tm_ctx** out);

/* Assembles K and the thermal load of one step on the device, then applies the
 * constraints (FEModel.assembleStep + applyConstraints). rhs_out (3*nn) may be NULL. */
tm_status tm_assemble_step(tm_ctx* ctx, const tm_step* step, double* rhs_out);

/* Loads a caller-assembled operator: the full symmetric 3x3-block CSR of
 * fullPatternFromUpper (09-assembly.js:136-148) with constraints already applied. */
tm_status tm_set_bcsr(tm_ctx* ctx, const int32_t* rowPtr, const int32_t* col, const double* val,
                      const uint8_t* isConstrained);

/* Solves K u = f for the current operator (LinearSolver.solve). The operator is
 * Jacobi-scaled in place on the first solve after an assembly, as in the reference. */
tm_status tm_solve(tm_ctx* ctx, const double* f, double* u, const tm_solve_opts* opts, tm_solve_info* info);
/* tm_solve with the displacement returned as float32 (3*nn floats), rounded to nearest on the
 * device: the step increment as the analysis keeps it (Float32Array.from(du),
 * src/core/11-analysis.js:256) and as the results file stores it (src/core/16-results-file.js),
 * with half the device-to-host bytes. */
tm_status tm_solve_f32(tm_ctx* ctx, const double* f, float* u32, const tm_solve_opts* opts, tm_solve_info* info);

/* y = K x with the current operator (unscaled before the first solve of a step). */
tm_status tm_matvec(tm_ctx* ctx, const double* x, double* y);

/* Downloads the current operator as the full block CSR of the mesh (for checks). */
tm_status tm_get_bcsr(tm_ctx* ctx, int32_t* rowPtr, int32_t* col, double* val);

/* Sizes: nn, ne, nnz blocks of the full block CSR, ndof, multigrid levels, coarsest dof. */
tm_status tm_sizes(tm_ctx* ctx, int64_t* out6);

tm_status tm_destroy(tm_ctx* ctx);

/* Message of the last error on this thread; returns its length. */
int32_t tm_last_error(char* buf, size_t len);

/* ---- device-resident entry points (inputs and outputs already in device memory) ---- */
/* tm_assemble_step with the load written to device memory (rhs_dev, 3*nn doubles, may be NULL). */
tm_status tm_assemble_step_device(tm_ctx* ctx, const tm_step* step, double* rhs_dev);
tm_status tm_solve_device(tm_ctx* ctx, const double* f_dev, double* u_dev, const tm_solve_opts* opts, tm_solve_info* info);
tm_status tm_matvec_device(tm_ctx* ctx, const double* x_dev, double* y_dev);
/* z = M^-1 r with the preconditioner the last solve built, in the solver's scaled space (the
 * reference's pc.apply(r, z), e.g. ICPC.apply, src/core/10-solver.js:784-798). */
tm_status tm_pc_apply(tm_ctx* ctx, const double* r, double* z);
tm_status tm_pc_apply_device(tm_ctx* ctx, const double* r_dev, double* z_dev);
/* Launch shapes the FP32 V-cycle's autotuner chose for the current hierarchy (no counterpart in
 * the reference, whose cycle runs on one thread): per shell level (fine to coarse) smoothed by column
 * sweeps, the warps per block of the sweep and of the residual kernel (2, 4 or 8; up to cap
 * levels written, *nlevels = all), and the stage count of the TMA level-0 sweep (0: not used).
 * TM_BAD_INPUT before a mixed-precision solve has run on this hierarchy. */
tm_status tm_vcycle_shapes(tm_ctx* ctx, int cap, int* nlevels, int* wpb_sweep, int* wpb_apply, int* tma_stages);
/* Fixes the FP32 V-cycle's launch shapes instead of timing them (e.g. shapes read back with
 * tm_vcycle_shapes on an earlier context of the same mesh): per swept shell level, fine to coarse
 * as tm_vcycle_shapes lists them, warps per block 2, 4 or 8 (levels beyond nlevels get 4);
 * tma_stages 2 or 3, or 0 for the planner's count (a count that does not fit falls back to it).
 * nlevels < 0 returns to autotuning. Takes effect at the next FP32 V-cycle; the shapes change
 * no arithmetic. */
tm_status tm_set_vcycle_shapes(tm_ctx* ctx, int nlevels, const int* wpb_sweep, const int* wpb_apply, int tma_stages);
/* The multigrid hierarchy built for the mesh (MultigridPC's levels, src/core/10-solver.js:620-662:
 * the solid level, buildShellLevel :248-335, then buildCoarseShellLevel :356-471 down to the
 * coarsest), for checks: per level, fine to coarse, 4 values (grid lines nx and ny of its
 * columns, nodes or aggregates nn, DOFs per node or aggregate b: 3 solid, 6 shell), up to cap
 * levels written into out4, *nlevels = all levels. */
tm_status tm_mg_levels(tm_ctx* ctx, int32_t cap, int32_t* out4, int32_t* nlevels);
/* Algorithmic bytes of the shell-level column sweeps of one FP32 V-cycle (no counterpart in the
 * reference; for the bandwidth figure of the sweeps): per swept shell level, 2 sweeps before and 2
 * after the coarse correction, each over all columns in 4 colours; a sweep reads the level's 6x6
 * blocks (36 floats and a column index each), the columns' explicit inverses, b and x and writes
 * x (the cycle's first colour launch on a level starts from x = 0 and reads neither its
 * columns' blocks nor their x), plus the column lists (24 bytes per column). *launches_per_cycle = the sweep launches of one cycle
 * (one per non-empty colour and sweep). Needs the multigrid hierarchy. */
tm_status tm_shell_sweep_bytes(tm_ctx* ctx, double* bytes_per_cycle, int32_t* launches_per_cycle);
/* The level-1 aggregate of every node (nn values): the solid-to-shell grouping of
 * buildShellLevel (src/core/10-solver.js:260-334) as the multigrid preconditioner uses it. */
tm_status tm_mg_node_agg(tm_ctx* ctx, int32_t* out);
/* CUDA-core fused multiply-add throughput of the current device in TFLOP/s, FP32 and FP64 (no
 * counterpart in the reference): the denominators of the compute roofline of the matrix-free level-0
 * kernels. Runs about a hundred milliseconds of arithmetic; either pointer may be NULL. */
tm_status tm_device_peaks(double* fp32_tflops, double* fp64_tflops);
/* Test hook of the timeout path (no counterpart in the reference). Every device wait of the library
 * is bounded: a wait that runs out makes the kernel flag the error, let its copies in flight land
 * and return, and the call fails with TM_TIMEOUT while the context stays usable. While on != 0,
 * the level-0 TMA sweep of the FP32 V-cycle (the assembled level-0 operator in mixed precision)
 * waits, with a short limit, for a stage flag that nothing sets, so that path can be exercised. */
tm_status tm_set_wait_test(tm_ctx* ctx, int32_t on);
/* Level-0 operator of the solves after the next tm_assemble_step (no counterpart in the reference,
 * whose LinearSolver always multiplies by the assembled matrix, 10-solver.js:933-994):
 * matrix_free = 0 (default) multiplies by the assembled 27-point stencil in the PCG apply and the
 * V-cycle's level-0 residuals and sweeps; 1 multiplies cell by cell with the element matrices of the
 * mesh's element classes (the level-0 sweep's column factors still come from the assembled diagonal
 * blocks). Both give the same operator up to the order of summation. The matrix-free path is taken
 * only where the mesh allows it (every cell's element classes in one table of at most 4095
 * combinations, columns of at most 128 nodes); tm_level0 reports the operator the current step uses. */
tm_status tm_set_level0(tm_ctx* ctx, int32_t matrix_free);
/* Drops the stored solutions of the warm start (a new LinearSolver's empty _warm list,
 * 10-solver.js:885-926): the next solve starts from zero. */
tm_status tm_clear_warm(tm_ctx* ctx);
tm_status tm_level0(tm_ctx* ctx, int32_t* matrix_free_active);

/* ---- element DOF histories at screening sites ---- */
/* Loads the per-step data that the DOF histories read (the shape matrices of every property set
 * and the element thermal loads) for step st without assembling the operator; tm_assemble_step
 * loads them too. */
tm_status tm_prepare_step(tm_ctx* ctx, const tm_step* st);
/* Adds to q (nel x 33: the 24 nodal DOFs then the 9 incompatible-mode amplitudes of every
 * listed element) the increment of the step loaded last (tm_prepare_step, tm_assemble_step), from that
 * step's displacement increment du (3*nn doubles): du at the element's nodes and
 * dalpha = K_aa^-1 (f_a - K_au du) (Model.accumulateStep with qOnly). The reference keeps du
 * of every step as Float32Array (src/core/11-analysis.js:256); the caller passes the values it
 * keeps. An element index < 0 (no element at that site) writes NaN into its row of q; an index
 * >= ne is TM_BAD_INPUT. Host pointers. */
tm_status tm_accumulate_q(tm_ctx* ctx, const double* du, int32_t nel, const int32_t* elems, double* q);
/* Engineering strain (6 per point, boxStrainAt order xx yy zz xy yz zx) of element elem[p] with
 * the element DOFs q[33 p ..] at the natural point nat[3 p ..] (each in [-1, 1], naturalCoords
 * of src/core/12-post.js:4-11). An element index < 0 gives NaN strains. Host pointers. */
tm_status tm_element_strains(tm_ctx* ctx, int32_t npts, const int32_t* elem, const double* q, const double* nat, double* eps);
/* The same with every array in device memory (element indices >= ne also give NaN rows). */
tm_status tm_accumulate_q_device(tm_ctx* ctx, const double* du_dev, int32_t nel, const int32_t* elems_dev, double* q_dev);
tm_status tm_element_strains_device(tm_ctx* ctx, int32_t npts, const int32_t* elem_dev, const double* q_dev,
                                    const double* nat_dev, double* eps_dev);

/* The transposes of the two steps from a step's displacement increment to the strain at a site,
 * for the adjoint of a function of the site strains (the peak bump dW; no counterpart in the
 * reference, whose tornado re-runs whole analyses):
 * tm_element_strains_adjoint: gq (33 per point) = B^T g, B the strain operator of
 * tm_element_strains at elem[p], nat[3 p ..] and g (6 per point) the function's derivative with
 * respect to the strains. tm_accumulate_q_adjoint: for the step loaded last (tm_prepare_step) and
 * gq (33 per element) the derivative with respect to the element DOF increment (du at the nodes,
 * dalpha = K_aa^-1 (f_a - K_au du)), gdu (24 per element) its derivative with respect to du at the
 * element's nodes and gA (one per element) its derivative with respect to the logarithm of the
 * thermal strain of the element's property set through dalpha. Host pointers. */
tm_status tm_element_strains_adjoint(tm_ctx* ctx, int32_t npts, const int32_t* elem, const double* nat, const double* g, double* gq);
tm_status tm_accumulate_q_adjoint(tm_ctx* ctx, int32_t nel, const int32_t* elems, const double* gq, double* gdu, double* gA);
/* The adjoint solve of the step assembled last for an adjoint load g (3*nn, the derivative of a
 * function with respect to the step's displacement increment u), and per property set m the
 * function's derivatives through that increment: dlogE[m] with respect to the logarithm of the set's
 * stiffness (lambda^T (f_m - K_m u)) and dlogA[m] with respect to the logarithm of its thermal strain
 * (lambda^T f_m), lambda = K^-1 g (the same MG-PCG; no counterpart in the reference). */
tm_status tm_adjoint_sensitivity(tm_ctx* ctx, const double* g, const double* u, const tm_solve_opts* opts, double* dlogE,
                                 double* dlogA, tm_solve_info* info);

/* ---- element stress histories ---- */
/* The sub-layers of the layered property sets for the step loaded last, which the stress
 * histories read (per sub-layer s of a section: sectionSubMeanD and sectionSubStress,
 * src/core/04-homogenize.js:196-204, and its z range, subLayerAt, src/core/09-assembly.js:547-552):
 * nsub per property set (0 for homogeneous sets, which use D and s0 of tm_step), then per
 * sub-layer in set order subZ (z0, z1), subD (36), subS0 (6). Call after tm_prepare_step or
 * tm_assemble_step for the same step. */
tm_status tm_set_sublayers(tm_ctx* ctx, const int32_t* nsub, const double* subZ, const double* subD, const double* subS0);
/* Model.accumulateStep without qOnly (src/core/09-assembly.js:508-544) over a list of
 * elements: state (stride doubles per element, stride >= 33 + 48 x the largest sub-layer count)
 * holds q (33), then per sub-layer the 7 strain-monomial stresses S_m (6 each) and the thermal
 * stress S_th (6); the step adds dq and, for born materials, D_m E_m(dq) and the step's thermal
 * stress increment. An element index < 0 writes NaN into its row. Host pointers. */
tm_status tm_accumulate_state(tm_ctx* ctx, const double* du, int32_t nel, const int32_t* elems, int32_t stride, double* state);
/* stateStress (src/core/09-assembly.js:555-571): engineering strain and stress (6 each) of
 * element elem[p] from its state (stride doubles per point) at the natural point nat[3 p ..];
 * NaN for an element index < 0. Host pointers. */
tm_status tm_state_stress(tm_ctx* ctx, int32_t npts, const int32_t* elem, const double* state, int32_t stride, const double* nat,
                          double* eps, double* sig);
/* The same with every array in device memory (element indices >= ne also give NaN rows). */
tm_status tm_accumulate_state_device(tm_ctx* ctx, const double* du_dev, int32_t nel, const int32_t* elems_dev, int32_t stride,
                                     double* state_dev);
tm_status tm_state_stress_device(tm_ctx* ctx, int32_t npts, const int32_t* elem_dev, const double* state_dev, int32_t stride,
                                 const double* nat_dev, double* eps_dev, double* sig_dev);

/* ---- field sampling ---- */
/* samplePlane: bilinear interpolation of component comp (0..2) of the nodal field u (3*nn
 * doubles) on mesh plane k at the points (x[p], y[p]); NaN where one of the four corner nodes
 * does not exist. Host pointers. */
tm_status tm_sample_plane(tm_ctx* ctx, const double* u, int32_t k, int32_t comp, int32_t npts, const double* x,
                          const double* y, double* out);
/* The same with u, x, y and out in device memory. */
tm_status tm_sample_plane_device(tm_ctx* ctx, const double* u_dev, int32_t k, int32_t comp, int32_t npts,
                                 const double* x_dev, const double* y_dev, double* out_dev);

/* ---- adjoint sensitivities (no counterpart in the reference, whose tornado charts re-run the
 * analysis per perturbed input, src/core/14-sensitivity.js) ---- */
/* For the solution u (3*nn, host) of the step assembled last: J = the mean squared residual of
 * the z displacements of the nodes of mesh plane k about their least-squares plane (a smooth
 * warpage measure), and per property set m its relative sensitivities dlogE[m] = dJ/dlog(E_m)
 * (the set's stiffness scaled, its thermal load with it) and dlogA[m] = dJ/dlog(alpha_m) (the
 * set's thermal strain scaled), from one adjoint solve K lambda = dJ/du with the solver and
 * preconditioner of tm_solve (opts as there; no warm start) and element sums. A material shared
 * by several sets has the sum over them. */
tm_status tm_warpage_sensitivity(tm_ctx* ctx, const double* u, int32_t k, const tm_solve_opts* opts, double* J, double* dlogE,
                                 double* dlogA, tm_solve_info* info);
/* After tm_warpage_sensitivity: dJ/dt_m per property set for one parameter t_m per set, whose
 * effect on the step's set data is given by dir (per set the derivatives of D and s0, or of W
 * and V for layered sets, with respect to t_m; NULL arrays are zero), e.g. a Poisson ratio's
 * dD/dnu and ds0/dnu. base is the step assembled last. The condensed element matrices are
 * differentiated by central differences of two condensations (relative step 1e-6), the rest
 * from the stored adjoint; the step's own element data are restored afterwards. */
tm_status tm_sensitivity_direction(tm_ctx* ctx, const tm_step* base, const tm_step* dir, double* dJ);

/* Runs the context's work on the caller's CUDA stream (a cudaStream_t) instead of its own
 * (the N-API addon passes the stream of the thread's device context). */
tm_status tm_set_stream(tm_ctx* ctx, void* stream);

/* ---- measurement (no counterpart in the reference, whose timings are nowMs() stamps,
 * src/core/11-analysis.js:192-203 and 10-solver.js:988) ---- */
/* Number of kernels this library has launched since it was loaded. */
int64_t tm_launch_count(void);
/* Kernel classes that the event timer can bracket. */
#define TM_K_APPLY0 0        /* level-0 stencil apply (fullMatVec) */
#define TM_K_SWEEP_SOLID 1   /* level-0 column smoother sweep of one colour (columnSweep, solid) */
#define TM_K_SWEEP_SHELL 2   /* shell-level column sweep of one colour (columnSweep, shell) */
#define TM_K_ASSEMBLE 3      /* stencil assembly (assembleStep) */
#define TM_K_GALERKIN01 4    /* Galerkin product solid -> shell (galerkinProduct) */
#define TM_K_APPLY_SHELL 5   /* shell-level residual (blockMatVec, b = 6) */
#define TM_K_SETUP_LEVEL0 6  /* multigrid set-up: level-0 column factors and transfer weights (factorColumns) */
#define TM_K_SETUP_SHELL 7   /* multigrid set-up: shell column factors, inverses and the Galerkin products between shells */
#define TM_K_SETUP_COARSEST 8 /* multigrid set-up: banded factor and explicit inverse of the coarsest level */
#define TM_K_TO_FP32 9       /* FP32 copies of the V-cycle's operators, factors and weights */
/* Brackets every following launch of one kernel class with CUDA events on the context's
 * stream (kernel = -1 switches the timer off); tm_kernel_timer_read returns the launches and
 * their summed device time since, and resets them. */
tm_status tm_kernel_timer(tm_ctx* ctx, int32_t kernel);
tm_status tm_kernel_timer_read(tm_ctx* ctx, int64_t* count, double* total_ms);

/* ---- Anand viscoplastic return map (13-fatigue.js:13-237) ---- */
typedef struct {
  double A, QR, xi, m, shat, n, h0, a, s0, nu;   /* Anand constants and Poisson ratio */
  const double* Etab;            /* E(T) in MPa on the 1 degC grid -80..300 (381 values) */
  const double* Ftab;            /* thermal strain F(T) on the same grid */
} tm_anand_material;

/* Screening of free-standing solder columns (screenJoints, 13-fatigue.js:379-455):
 *   table: nsites x ntemps x 6 bump-layer total strains at the cycling temperatures temps;
 *   the time history (t, T, cycle, phase) of cycleHistory (13-fatigue.js:275-293);
 * outputs per site: dW (inelastic work density of the last cycle), dE (equivalent
 * inelastic strain of the last cycle), stab (cycle-to-cycle change). Sites whose
 * first table entry is not finite are skipped (NaN outputs). Host pointers. */
tm_status tm_anand_screen(const tm_anand_material* mat, int32_t nsites, int32_t ntemps, const double* temps,
                          const double* table, int32_t nsteps, const double* t, const double* T,
                          const int32_t* cycle, const int32_t* phase, int32_t cycles,
                          double* dW, double* dE, double* stab);

/* The same with device pointers for table and outputs (time history on the host). */
tm_status tm_anand_screen_device(const tm_anand_material* mat, int32_t nsites, int32_t ntemps, const double* temps,
                                 const double* table_dev, int32_t nsteps, const double* t, const double* T,
                                 const int32_t* cycle, const int32_t* phase, int32_t cycles,
                                 double* dW_dev, double* dE_dev, double* stab_dev);

/* An elastic pillar under each solder joint (a DDI microbump: solder cap on a Cu pillar). */
typedef struct {
  double fs;                     /* solder height fraction of the joint, 1 - pillarH / standoff, in (0, 1] */
  double nu;                     /* pillar Poisson ratio */
  const double* Etab;            /* pillar E(T) in MPa on the 1 degC grid -80..300 (381 values) */
  const double* Ftab;            /* pillar thermal strain F(T) on the same grid */
} tm_pillar;

/* tm_anand_screen for joints that are a solder cap on an elastic pillar (screenDdi): per time
 * step the column-average axial and shear strains of the layer (less the thermal strains of cap
 * and pillar) are prescribed, the cap and the pillar carry the same axial and shear stresses
 * and the cap's in-plane stresses vanish (stepSeriesColumn). Host pointers. */
tm_status tm_anand_screen_pillar(const tm_anand_material* mat, const tm_pillar* pillar, int32_t nsites, int32_t ntemps,
                                 const double* temps, const double* table, int32_t nsteps, const double* t, const double* T,
                                 const int32_t* cycle, const int32_t* phase, int32_t cycles,
                                 double* dW, double* dE, double* stab);
/* The same with device pointers for table and outputs (time history and tables on the host). */
tm_status tm_anand_screen_pillar_device(const tm_anand_material* mat, const tm_pillar* pillar, int32_t nsites, int32_t ntemps,
                                        const double* temps, const double* table_dev, int32_t nsteps, const double* t,
                                        const double* T, const int32_t* cycle, const int32_t* phase, int32_t cycles,
                                        double* dW_dev, double* dE_dev, double* stab_dev);

/* Screening that allocates no device memory (no counterpart in the reference). For callers that
 * cannot call cudaMalloc while they screen: a host application whose allocator already owns the
 * device memory (a caching allocator, a process held to a fixed memory budget), or one that
 * forbids allocations after start-up because cudaMalloc and cudaFree synchronize the device.
 * The per-step tables live in a fixed array of the library (TM_NOALLOC_MAX_STEPS steps and
 * TM_NOALLOC_MAX_TEMPS cycling temperatures at most, about 360 KB), which every GPU that loads
 * the library holds until the process exits; larger inputs are refused with TM_BAD_INPUT.
 * The caller passes the strain table and the three outputs in device memory (nsites doubles
 * each) and the time history, temperatures and material tables on the host; stream may be NULL.
 * The first call on a device looks up the array's device address (cudaGetSymbolAddress) with
 * that device current; make that first call before any stream capture. Every call shares the
 * array and overwrites it: calls that overlap on the GPU (other threads, other streams) race. */
#define TM_NOALLOC_MAX_STEPS 4096
#define TM_NOALLOC_MAX_TEMPS 512
tm_status tm_anand_screen_noalloc(const tm_anand_material* mat, int32_t nsites, int32_t ntemps, const double* temps,
                                  const double* table_dev, int32_t nsteps, const double* t, const double* T,
                                  const int32_t* cycle, const int32_t* phase, int32_t cycles,
                                  double* dW_dev, double* dE_dev, double* stab_dev, void* stream);

/* ---- bump submodel (BumpSubmodel, src/core/13-fatigue.js:470-1104) ---- */
/* One pitch cell around a bump: B-bar hexes on the grid xs x ys x zs with a material per cell
 * (0 substrate slice, 1 solder, 2 underfill, 3 silicon; cells in (i, j, k) order, k fastest),
 * Anand solder Gauss points (elastic ones when elasticSolder), the other parts incremental
 * elastic. The cut boundary (the nodes on the six faces, ascending node id (i ny + j) nz + k)
 * moves with the global displacement fields (prescribe / fieldAt): for boundary node q its 8
 * global nodes bGlob[8q..] (indices into the nglob global nodes the caller passes) and the
 * trilinear weights bW[8q..]; the global fields at the nt ascending global temperatures ts
 * (fields: nt x nglob x 3) and at 25 degC (u25). Material tables on the 1 degC grid -80..300
 * (381 points): solder E and F in `solder`, underfill E/F and Poisson ratio, silicon F and its
 * stiffness siD (36), substrate slice D (381 x 36) and F (381 x 3). nuMax: NU_MAX_SUBMODEL.
 * zt / zaf: the pad and UBM heights that bound the two averaging layers (SUB_T_AVG). */
typedef struct {
  int32_t nx, ny, nz;
  const double *xs, *ys, *zs;
  const int32_t* cellMat;
  int32_t nglob, nt;
  const double* ts;
  const double* fields;
  const double* u25;
  int32_t nb;
  const int32_t* bGlob;
  const double* bW;
  tm_anand_material solder;
  int32_t elasticSolder;
  const double* ufE;
  const double* ufF;
  double ufNu;
  const double* siD;
  const double* siF;
  const double* subD;
  const double* subF;
  double nuMax, zt, zaf;
  /* homogenized-layer consistency mode, BumpSubmodel opts.uniformMaterial (13-fatigue.js:538,
   * 556, 711-748, 757; the V7 check), 0: off. The bump layer's solder and underfill cells become
   * one material: solder columns (columnD) and underfill (isoD clamped at nuMaxGlobal) with
   * volume fractions density and 1 - density. Every substrate element layer takes the step-mean
   * stiffness of the top substrate band's sub-layer at its mid-height, with the band's
   * through-thickness response (Voigt thickness modulus, Turner-weighted thermal strain). The band
   * section (buildBandSection, 04-homogenize.js:139-183): nsec sub-layers, secZ (z0, z1 per
   * sub-layer, ascending), secD (36 x TGRID_N per sub-layer: its shell stiffness table), secF
   * (3 x TGRID_N per sub-layer: its thermal strain table). There are no Anand points in this
   * mode: tm_submodel_step works, tm_submodel_run refuses. */
  int32_t uniformMaterial;
  double density, nuMaxGlobal;
  int32_t nsec;
  const double* secZ;
  const double* secD;
  const double* secF;
} tm_submodel_spec;
typedef struct tm_sub tm_sub;
tm_status tm_submodel_create(const tm_submodel_spec* spec, tm_sub** out);
/* Preconditioner of the Newton steps' inner PCG solves: TM_SUB_PC_IC, the reference's IC(0)
 * (_solve, 13-fatigue.js:886-917; the default), or TM_SUB_PC_LINE, a z-line block Jacobi (the
 * cell's node columns' 3x3-block tridiagonal parts factored exactly; one launch per apply, where
 * IC(0) runs one launch per level set). The inner solves stop at the same relative residual
 * either way, so the Newton iterates agree to that tolerance. */
#define TM_SUB_PC_IC 0
#define TM_SUB_PC_LINE 1
tm_status tm_submodel_set_precond(tm_sub* sm, int32_t kind);
/* Work counters of the submodel so far: inner solves, and their PCG iterations summed. */
tm_status tm_submodel_counters(tm_sub* sm, int64_t* out2);
tm_status tm_submodel_destroy(tm_sub* sm);
/* nn, ne, boundary nodes, solder Gauss points */
tm_status tm_submodel_sizes(tm_sub* sm, int64_t* out4);
/* stepTo(T, dt) (13-fatigue.js:924-956): Newton to temperature T; converged (0/1), Newton
 * iterations and the largest plastic increment of the solder points. */
tm_status tm_submodel_step(tm_sub* sm, double T, double dt, int32_t* converged, int32_t* newton, double* dMax);
/* The displacement (3 nn) and the solder points' W and ebar (element-major; NULL to skip). */
tm_status tm_submodel_get(tm_sub* sm, double* u, double* W, double* ebar);
/* run (13-fatigue.js:1004-1104) over the cycle history (t, T, cycle of cycleHistory) with
 * adaptive sub-steps: out (10) = dW, dWdie, dWsub, dE, dEdie, dEsub, stabChange, steps,
 * cutbacks, newtonPerStep; perCycle (2 per cycle) = dWdie, dWsub; loop (4 per history point) =
 * tau, gamma of the die-side layer and of the substrate-side layer along (cphi, sphi), the
 * site's direction from the die centre. A step that fails after 8 cutbacks is TM_NOT_CONVERGED. */
tm_status tm_submodel_run(tm_sub* sm, int32_t nsteps, const double* t, const double* T, const int32_t* cycle, int32_t cycles,
                          double cphi, double sphi, double* out10, double* perCycle, double* loop);
/* tm_submodel_run with the result's section record (13-fatigue.js:1053-1078, 1098-1101): phase
 * (per history point, cycleHistory's phase) marks the ramps and dwells; at the end of each of
 * them in the last cycle a stress snapshot is taken. *nSnaps counts them; up to maxSnaps are
 * written: snapMeta (4 each: T, t, cycle, phase) and snapSig (48 floats per element each). */
tm_status tm_submodel_run_sections(tm_sub* sm, int32_t nsteps, const double* t, const double* T, const int32_t* cycle,
                                   const int32_t* phase, int32_t cycles, double cphi, double sphi, double* out10, double* perCycle,
                                   double* loop, int32_t maxSnaps, int32_t* nSnaps, double* snapMeta, float* snapSig);
/* _stressSnapshot (13-fatigue.js:965-989) of the current state at temperature T: per element the
 * 8 nodes' 6 stresses (float32), extrapolated from the Gauss points (GP_TO_NODE). */
tm_status tm_submodel_stress_snapshot(tm_sub* sm, double T, float* out);

/* n submodels over the same history at once (the screened sites of a die): out10, perCycle
 * and loop hold n consecutive records; status[i] is each run's status (TM_OK or the failure),
 * and the call returns the first failure. The submodels advance together in groups of up to 64:
 * each phase of their Newton steps (boundary, assembly and gathers, norms, the inner solves'
 * products, reductions and preconditioner, commits) is one launch over every submodel in that
 * phase, while each keeps its own sub-steps, cutbacks and Newton iterations; a submodel's result
 * equals its tm_submodel_run result with the same preconditioner. */
tm_status tm_submodel_run_batch(int32_t n, tm_sub* const* subs, int32_t nsteps, const double* t, const double* T,
                                const int32_t* cycle, int32_t cycles, const double* cphi, const double* sphi, double* out10,
                                double* perCycle, double* loop, int32_t* status);

/* Batched material-point steps: npts independent points, each with a 12-double state
 * (ep[6], s, ebar, W, sigEq, lastD, spare) updated in place when commit != 0;
 * eps (6 per point) engineering mechanical strain; sig (6 per point) and, when
 * D != NULL, the consistent tangent (36 per point). Host pointers. */
tm_status tm_anand_step(const tm_anand_material* mat, int32_t npts, double* state, const double* eps,
                        double T, double dt, double* sig, double* D, int32_t commit);

/* One site of screenJoints' loop (13-fatigue.js:416-451; with a pillar, screenDdi's stepSeriesColumn)
 * and the derivatives of its last-cycle dW and dE with respect to every entry of its strain table
 * (table: ntemps x 6, gW and gE the same shape), for the adjoint of the peak bump dW (no counterpart
 * in the reference, whose tornado re-runs whole analyses). Forward mode: each table entry is a
 * direction carried through the whole history, iterations included, so the result is the exact
 * derivative of the screening as computed. pillar may be NULL (a free-standing column). */
tm_status tm_anand_screen_gradient(const tm_anand_material* mat, const tm_pillar* pillar, int32_t ntemps, const double* temps,
                                   const double* table, int32_t nsteps, const double* t, const double* T, const int32_t* cycle,
                                   const int32_t* phase, int32_t cycles, double* dW, double* dE, double* gW, double* gE);

#ifdef __cplusplus
}
#endif

#endif /* TMSOLVE_H */
