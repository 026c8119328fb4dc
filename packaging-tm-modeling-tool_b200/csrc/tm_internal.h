// Internal declarations of the B200 solve-path library (not part of the C-ABI).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "../../include/tmsolve.h"

namespace tmg {

// ---- error handling --------------------------------------------------------------------
struct Error {
  tm_status status;
  std::string msg;
};
[[noreturn]] void fail(tm_status st, const std::string& msg);
void set_last_error(const std::string& msg);
void cuda_check(cudaError_t e, const char* what);
void require_device();   // TM_NO_DEVICE unless the current device is an sm_100 GPU
#define TM_CUDA_CHECK(x) ::tmg::cuda_check((x), #x)

// ---- device buffers ---------------------------------------------------------------------
template <class T>
struct DBuf {
  T* p = nullptr;
  size_t n = 0;
  DBuf() = default;
  DBuf(const DBuf&) = delete;
  DBuf& operator=(const DBuf&) = delete;
  ~DBuf() { release(); }
  void alloc(size_t count) {
    if (count == n && p) return;
    release();
    n = count;
    if (count) TM_CUDA_CHECK(cudaMalloc((void**)&p, count * sizeof(T) + 16));
  }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
  }
  void upload(const T* h, size_t count, cudaStream_t s) {
    alloc(count);
    if (count) TM_CUDA_CHECK(cudaMemcpyAsync(p, h, count * sizeof(T), cudaMemcpyHostToDevice, s));
  }
  void upload(const std::vector<T>& v, cudaStream_t s) { upload(v.data(), v.size(), s); }
  void zero(cudaStream_t s) {
    if (n) TM_CUDA_CHECK(cudaMemsetAsync(p, 0, n * sizeof(T), s));
  }
  void download(T* h, size_t count, cudaStream_t s) const {
    if (count) TM_CUDA_CHECK(cudaMemcpyAsync(h, p, count * sizeof(T), cudaMemcpyDeviceToHost, s));
  }
};

// launch shape of the level-0 panel smoother: threads per CTA (also the node capacity of a
// column panel), the resident CTAs per SM its register budget is sized for
// (FP32 and FP64 builds of the kernel) and the unroll depth of its 27-slot residual loop
#ifndef TM_PANEL_THREADS
#define TM_PANEL_THREADS 256
#endif
#ifndef TM_PANEL_MINB
#define TM_PANEL_MINB 8
#endif
#ifndef TM_PANEL_MINB_F64
#define TM_PANEL_MINB_F64 6
#endif
#ifndef TM_PANEL_UNROLL
#define TM_PANEL_UNROLL 3
#endif
// FP32 level-0 apply: positions per thread (1, 2 or 4; the operator rows are padded to a
// multiple of 4), unroll depth of its slot loop and the resident CTAs its registers are sized for
#ifndef TM_SWEEP_TMA
#define TM_SWEEP_TMA 1
#endif
#ifndef TM_APPLY32_NPT
#define TM_APPLY32_NPT 2
#endif
#ifndef TM_APPLY32_UNROLL
#define TM_APPLY32_UNROLL 3
#endif
#ifndef TM_APPLY32_MINB
#define TM_APPLY32_MINB 10
#endif
// level-0 operator from the cell-class table (tm_mf.cu) instead of the assembled stencil, for
// operators assembled by tm_assemble_step (0: the assembled stencil everywhere)
#ifndef TM_MATRIX_FREE
#define TM_MATRIX_FREE 1
#endif
#define TM_STR_(x) #x
#define TM_UNROLL(n) _Pragma(TM_STR_(unroll n))

// number of stencil slots of a node: offsets (di, dj, dk) in {-1,0,1}^3, slot = (di+1)*9+(dj+1)*3+(dk+1);
// ascending slot order is ascending neighbour node id (nodes are numbered z fastest, then y, then x)
constexpr int NSLOT = 27;
constexpr int SLOT_SELF = 13;
constexpr int SLOT_DOWN = 12;  // (0, 0, -1): the node below in the same column

// ---- multigrid shell level (6 DOFs per aggregate) ------------------------------------------
// IC(0) of the scaled level-0 operator (ICPC, 10-solver.js:719-800): the scalar upper CSR of the
// block pattern (rows 3i+p, columns j >= i with q >= p on the diagonal block, sorted), for every
// entry its index into the slot-major operator, the column lists of U (rows i < c with U(i, c),
// ascending, and the entry's position) and the node level schedules of the factorization /
// forward solve (levels of increasing node ids) and of the backward solve
struct IcFactor {
  long long epoch = -1;                // structure built for this hierarchy epoch
  int n = 0;
  long long nnz = 0;
  DBuf<int> d_rowPtr, d_col, d_gmap, d_tStart, d_tRow, d_tPos;
  DBuf<int> d_fwdNodes, d_bwdNodes;
  std::vector<int> fwdStart, bwdStart;
  DBuf<double> d_U;
  DBuf<int> d_fail;
  double shift = 0;
  bool ready = false;
  // the level launches of one apply as a CUDA graph, for the (r, z, stream) it was captured with
  cudaGraphExec_t exec = nullptr;
  const double* gr = nullptr;
  double* gz = nullptr;
  cudaStream_t gst = nullptr;
  void drop_graph() {
    if (exec) cudaGraphExecDestroy(exec);
    exec = nullptr; gr = nullptr; gz = nullptr; gst = nullptr;
  }
  ~IcFactor() { drop_graph(); }
};

struct ShellLevel {
  int nx = 0, ny = 0, nn = 0;          // columns nx*ny, aggregates nn
  int wpbSweep = 4, wpbApply = 4;      // warps per block of the FP32 sweep and residual (autotuned)
  std::vector<double> xs, ys;          // grid lines of the level's columns
  std::vector<int> colStart;           // nx*ny+1
  std::vector<double> zref, zlo, zhi;  // per aggregate
  std::vector<int> keepX, keepY;
  bool hasKeep = false;
  // operator: block CSR with 6x6 blocks, pattern fixed by the mesh
  std::vector<int> rowPtr, col, diag;
  int nb = 0;
  DBuf<int> d_rowPtr, d_col;
  DBuf<double> d_val;                  // 36*nb
  DBuf<float> d_val32;                 // mixed precision copy
  // dense per-column factors and the explicit inverses of the column blocks
  std::vector<long long> cfPtr;        // ncol+1 (offsets in doubles)
  DBuf<long long> d_cfPtr;
  DBuf<double> d_cf, d_cfInv;
  DBuf<float> d_cfInv32;
  DBuf<int> d_colStart;
  int maxm = 0;                        // largest column size in DOFs
  int maxColBlocks = 0;                // most blocks in the rows of one column
  // colours: columns with (i%2, j%2) = colour, as lists
  DBuf<int> d_colorCols[4];
  int colorCount[4] = {0, 0, 0, 0};
  // per column (all columns, and per colour list entry): first and one-past-last aggregate and
  // block, and the offset of the column's inverse block
  DBuf<int4> d_colMeta, d_colorMeta[4];
  DBuf<long long> d_colorCf[4];
  // prolongation from the next (coarser) level to this one: per aggregate f of this level
  // parents idx with 6x6 weights (buildCoarseShellLevel, 10-solver.js:396-471)
  std::vector<int> prolPtr, prolIdx;
  std::vector<double> prolW;
  DBuf<int> d_prolPtr, d_prolIdx;
  DBuf<double> d_prolW;
  // children of the next level's aggregates (transposeProl)
  std::vector<int> chPtr, chIdx, chW;
  DBuf<int> d_chPtr, d_chIdx, d_chW;
  // Galerkin contributions into this level's blocks from the finer shell level: per block a list
  // of (fine block, weight entry of the row child, weight entry of the column child) triples
  DBuf<int> d_galStart, d_galList;
  // Galerkin pattern bookkeeping for this level as a coarse level: max blocks per row
  int maxRowBlocks = 0;
  // work vectors
  DBuf<double> d_b, d_x, d_res;
  DBuf<float> d_prolW32, d_b32, d_x32, d_res32;
  // coarsest level: banded factor and explicit inverse
  bool coarsest = false;
  int bandBw = 0, denseN = 0;
  DBuf<double> d_band;                 // denseN*(bw+1): the operator's lower band, then its Schur complements
  DBuf<double> d_bandL;                // denseN*(bw+1): the banded Cholesky factor
  DBuf<double> d_bandLt;               // denseN*(bw+1): its transpose, row i holding L[i..i+bw][i]
  DBuf<double> d_dinv;                 // inverses of the factor's 32x32 diagonal blocks
  DBuf<double> d_jit;                  // pivot floor of the factor
  DBuf<double> d_inv;                  // denseN*denseN
  DBuf<float> d_inv32;
};

struct Context {
  int dev = 0;
  int nnp = 0;                         // row stride of the slot-major level-0 arrays
  cudaStream_t stream = nullptr;
  // mesh (host copies of what the structure builders need)
  int nx = 0, ny = 0, nz = 0, nn = 0, ne = 0, npset = 0, ngroups = 0;
  std::vector<double> xs, ys, zs, coords;
  std::vector<int> nodeId, conn, eIJK, colStart, cellElems, eGroup, ePset, groupStage, constr, featureX, featureY;
  std::vector<int8_t> ePart;
  std::vector<double> eScale;
  std::vector<int> nodeIJK;            // 3*nn
  // stencil structure
  std::vector<int> nbr;                // 27*nn, slot-major
  std::vector<int> slotMask;           // nn: bit s set when (n, nbr[s]) share an element (the block CSR pattern)
  // device copies of the level-0 arrays are stored in colour-major position order: the nodes of all
  // colour-0 columns first (columns in ascending order, each column contiguous), then colour 1, ...
  // so that one colour's sweep streams a contiguous block; pos[n] is the position of node n
  std::vector<int> pos, posNode;
  DBuf<int> d_pos, d_posNode;
  DBuf<int> d_nbr, d_slotMask, d_nodeIJK, d_cellElems, d_eGroup, d_groupStage, d_eClass, d_colStart, d_constr;
  DBuf<double> d_eScale;
  // element classes: (property set, hx, hy, hz)
  int ncls = 0;
  std::vector<int> eClass, clsPset;
  std::vector<double> clsH;            // 3*ncls
  DBuf<int> d_clsPset;
  DBuf<double> d_clsH, d_clsKc, d_clsFc;   // 576, 24 per class
  DBuf<int> d_clsBorn;
  DBuf<double> d_psetM;                // 6*1089 per property set
  DBuf<double> d_clsF33;               // 33 per class: uncondensed element thermal load (elementFth)
  DBuf<int> d_psetLayered, d_psetBorn;
  // matrix-free level 0 (tm_mf.cu): per mesh cell one cell class (the (class, scale) pairs of its
  // elements) whose combined condensed matrix is formed per step; per DOF the gather scale gs (S,
  // zero at constrained DOFs), the row scale os (S) and the kept diagonal cd of constrained rows
  bool mf = false;                     // level 0 is applied from the cell-class table (operator from tm_assemble_step)
  bool mfBuilt = false, mfAvailable = false, mfModule = false;
  int mfStage = 0;                     // stage the cell classes were built for (element birth scales)
  int ncc = 0;
  DBuf<uint16_t> d_cellCls;            // per cell, 0xFFFF: no element
  DBuf<int> d_ccInfo;                  // per cell class: the element classes (second -1 when single)
  DBuf<double> d_ccScale;              // per cell class: the elements' assembly scales
  DBuf<double> d_ccK;                  // 576 per cell class
  DBuf<float> d_ccK32;
  DBuf<double> d_gs, d_os, d_cd;
  DBuf<float> d_gs32, d_os32, d_cd32;
  DBuf<int> d_colP0;                   // per node column: position of its first node (-1: empty)
  IcFactor ic;                         // the IC(0) preconditioner (tm_ic0.cu)
  int pcKind = -1;                     // kind of the preconditioner built last (TM_PC_*)
  bool stepReady = false;              // shape matrices and thermal loads of an assembled step are on the device
  DBuf<double> d_stepD, d_stepS0;      // the step's homogeneous D (36) and s0 (6) per property set
  // sub-layers of the layered sets for the stress histories (tm_set_sublayers): offsets per set,
  // z ranges (2), step-mean stiffness (36) and thermal stress increment (6) per sub-layer
  bool subReady = false;
  int maxSub = 1;
  DBuf<int> d_subOff;
  DBuf<double> d_subZ, d_subD, d_subS0;
  DBuf<int> d_eIJK;
  DBuf<double> d_zs;
  DBuf<float> d_u32out;                // float32 copy of a solution (tm_solve_f32)
  DBuf<double> d_sensU, d_sensLam;     // solution and adjoint of tm_warpage_sensitivity
  bool sensReady = false;
  DBuf<int> d_conn;                    // 8*ne, uploaded on first use by the DOF-history entry points
  DBuf<double> d_xs, d_ys;             // mesh lines and the node index grid, uploaded on first use
  DBuf<int> d_nodeId;                  // by the plane sampler
  // operator (level 0): 243 values per position, slot-major ((s*9 + v)*nnp + p), and its FP32
  // copy; the slot-major device arrays (operator, neighbour ids) use the row stride nnp (nn
  // rounded up to a multiple of 4; zero values and id -1 in the padding), so that adjacent
  // positions of the FP32 operator load as one 8- or 16-byte vector
  DBuf<double> d_val;
  DBuf<float> d_val32;
  DBuf<double> d_rhs;
  DBuf<uint8_t> d_isC;
  std::vector<uint8_t> isC;
  int stage = 0;
  bool assembled = false, scaled = false, fp32Ready = false, mgFp32 = false;
  // solver state
  DBuf<double> d_s, d_f, d_uio, d_bs, d_x, d_r, d_z, d_p, d_q, d_tmp, d_tmp2;
  DBuf<double> d_partial, d_scalars;
  DBuf<uintptr_t> d_mdPtr;             // vector tables of the batched dot products
  DBuf<double> d_mdPart, d_warmKV;     // their partial sums; K times the warm-start basis
  DBuf<int> d_jitter;
  // level 0 smoother and transfer
  DBuf<double> d_F;                    // 18 per node (column block-tridiagonal factors)
  DBuf<int> d_colorCols[4];
  int colorCount[4] = {0, 0, 0, 0};
  int maxColLen = 0;
  // level-0 sweep of the FP32 V-cycle with TMA-streamed operator rows (tm_sweep_tma.cu): per
  // colour the runs of whole columns of each CTA (indices into the colour's column list), the
  // longest run, the chunk stages, the two tensor maps (operator rows, neighbour ids)
  bool tsReady = false;
  long long tunedEpoch = -1;           // hierarchy epoch the FP32 V-cycle's launch shapes were tuned for
  long long shapeEpoch = 0;            // bumped when the launch shapes change (the cycle is captured again)
  int tsPlanned = 0;                   // the largest TMA stage count that fits (the planner's)
  bool shapesPinned = false;           // the caller fixed the shapes (tm_set_vcycle_shapes): no timing
  std::vector<int> pinSweep, pinApply; // pinned warps per block per swept shell level
  int pinStages = 0;                   // pinned TMA stage count (0: the planner's)
  int tsParts = 0, tsMaxNodes = 0, tsStages = 0;
  DBuf<int> d_tsPart[4];
  DBuf<float> d_val32p;                // position-major FP32 operator (243 values per position)
  DBuf<int> d_nbrp;                    // position-major neighbour ids (27 per position)
  DBuf<int> d_err;                     // set by a bounded device wait that ran out
  bool level0Mf = false;               // caller's choice of the level-0 operator (tm_set_level0)
  bool waitTest = false;               // test hook: the TMA sweep waits for a stage flag that nothing sets
  // level-0 column panels: the columns of one colour packed into groups of at most panelCap nodes,
  // one CTA per group (group g holds colour columns grpStart[g] .. grpStart[g+1]-1); colPos holds
  // the position of the first node of every colour column plus one past the colour's last node
  int panelCap = TM_PANEL_THREADS, panelMaxCols = 0;
  DBuf<int> d_grpStart[4], d_colPos[4];
  int colourPos[5] = {0, 0, 0, 0, 0};  // colour k occupies positions colourPos[k] .. colourPos[k+1]-1
  int grpCount[4] = {0, 0, 0, 0};
  std::vector<int> nodeAgg, aggPtr, aggNodes;   // level 0 -> 1 (nodeAgg -1: a held node of a module stage)
  std::vector<double> zp;              // z of node minus zref of its aggregate
  DBuf<int> d_nodeAgg, d_aggPtr, d_aggNodes;
  // stacked-module stages (09-assembly.js:397-443): the constraints of those stages (the package's
  // 3-2-1 plus each module's own), and for the stage assembled last its born elements and the nodes
  // they touch (empty outside module stages); the hierarchy is built for activeKey (0: the whole package)
  std::vector<int> modConstr, meshConstr;
  std::vector<uint8_t> actElem, actNode;
  int activeKey = 0, hierKey = 0;
  bool moduleStage = false;            // the step assembled last is a stacked-module stage (unborn elements skipped)
  // Galerkin contributions of the solid operator to the level-1 blocks: per block the
  // (position, slot) pairs, coded position*27 + slot, in (slot, position) order
  DBuf<int> d_g01Start, d_g01List;
  DBuf<double> d_zp, d_W01;            // 18 per node
  int maxRowBlocks1 = 0;
  DBuf<double> d_res0;                 // level-0 residual
  DBuf<float> d_F32, d_W01_32, d_res0_32;
  // FP32 inner solve of the mixed-precision refinement
  DBuf<float> d_r32, d_z32, d_p32, d_q32, d_d32;
  // caller stream, launch counter and the event timer of one kernel class
  bool ownStream = true;
  int timerKernel = -1;
  std::vector<std::pair<cudaEvent_t, cudaEvent_t>> timerEvents;
  std::vector<ShellLevel*> shells;     // levels 1..L-1
  bool hierarchy = false;
  bool pcReady = false;
  long long pcKey = -1;
  bool needRebuild = true;
  double ratePerDecade = 0;
  int colJitter = 0, shellJitter = 0;
  // warm start basis (unscaled space)
  std::vector<DBuf<double>*> basis;
  // the V-cycle as a CUDA graph per precision (0: FP64, 1: FP32), captured on first use on a
  // private stream and replayed on the caller's; captured again when its vectors or the
  // hierarchy's buffers (structEpoch) change
  cudaGraphExec_t vcGraph[2] = {nullptr, nullptr};
  size_t vcKey[2] = {0, 0};
  long long vcNodes[2] = {0, 0};
  cudaStream_t capStream = nullptr;
  long long structEpoch = 0;
  ~Context();
};

// ---- host structure builders (tm_hierarchy.cpp) ----------------------------------------------
void build_stencil(Context& c);
void build_classes(Context& c);
void build_hierarchy(Context& c);

// ---- set-up kernels (tm_setup.cu, compiled without fused multiply-add) -----------------------
void launch_shape_matrices(Context& c, const tm_step& st);
void launch_class_condense(Context& c);
void launch_assemble(Context& c);
void launch_constraints(Context& c);
void launch_scale(Context& c);
void launch_scale_rhs(Context& c, const double* f, double* bs);
void launch_factor_columns(Context& c);
void launch_w01(Context& c);
void launch_galerkin01(Context& c);
void launch_galerkin_shell(Context& c, int l);
void launch_factor_shell(Context& c, ShellLevel& L);
void launch_factor_coarsest(Context& c, ShellLevel& L);
void launch_to_fp32(Context& c);
// element DOF histories and strains at points (device pointers; elems/elem, q, nat, eps on the device)
void launch_accumulate_q(Context& c, const double* du, int nel, const int* elems, double* q);
void launch_element_strains(Context& c, int np, const int* elem, const double* q, const double* nat, double* eps);
void launch_element_strains_adjoint(Context& c, int np, const int* elem, const double* nat, const double* g, double* gq);
void launch_accumulate_q_adjoint(Context& c, int nel, const int* elems, const double* gq, double* gdu, double* gA);
void launch_sample_plane(Context& c, const double* u, int k, int comp, int npts, const double* x, const double* y, double* out);
void launch_accumulate_state(Context& c, const double* du, int nel, const int* elems, int stride, double* state);
void launch_sens(Context& c, const double* u, const double* lam, double* outHost);
void sens_direction(Context& c, const tm_step& base, const tm_step& dir, const double* u, const double* lam, double* dJ);
void launch_state_stress(Context& c, int np, const int* elem, const double* state, int stride, const double* nat, double* eps,
                         double* sig);

// ---- IC(0) (tm_ic0.cu) -------------------------------------------------------------------------
void build_ic(Context& c);                                   // structure (once) + shifted factorization
void launch_ic_apply(Context& c, const double* r, double* z);
// the same on any node-block pattern (the bump submodel's tangent)
void ic_build_structure(IcFactor& F, int nn, const std::vector<int>& nrp, const std::vector<int>& ncol,
                        const std::vector<long long>& vbase, long long vstride, cudaStream_t st);
void ic_factor(IcFactor& F, const double* val, cudaStream_t st);
void ic_apply(IcFactor& F, const double* r, double* z, cudaStream_t st);

// ---- launch accounting ------------------------------------------------------------------------
enum KernelId {
  K_APPLY0 = 0, K_SWEEP_SOLID = 1, K_SWEEP_SHELL = 2, K_ASSEMBLE = 3, K_GALERKIN01 = 4, K_APPLY_SHELL = 5,
  K_SETUP_LEVEL0 = 6, K_SETUP_SHELL = 7, K_SETUP_COARSEST = 8, K_TO_FP32 = 9, K_NKERNEL
};
void note_launch(int count = 1);
struct TimedLaunch {   // brackets one launch with events when the context times this kernel class
  Context& c;
  bool on;
  cudaEvent_t a = nullptr, b = nullptr;
  TimedLaunch(Context& ctx, int kid);
  ~TimedLaunch();
};

// ---- solve kernels (tm_solve.cu) -------------------------------------------------------------
void launch_apply0(Context& c, const double* x, double* y, const double* b);   // y = K x, or b - K x when b != nullptr
void launch_apply0_f32(Context& c, const double* x, double* y, const double* b);
void launch_dot(Context& c, const double* a, const double* b, size_t n, double* out_dev);
// every dot a_i . b_j (n entries) into out[i * b.size() + j] on the host: one launch pair and one
// synchronization per 512 pairs
void multi_dot_host(Context& c, const std::vector<const double*>& a, const std::vector<const double*>& b, size_t n, double* out);
void launch_axpy2(Context& c, const double* alpha_dev, const double* p, double* x, const double* q, double* r, size_t n);
void launch_xpby(Context& c, const double* z, const double* beta_dev, double* p, size_t n);
void launch_zero_constrained(Context& c, double* v);
void launch_vcycle(Context& c, const double* r, double* z, bool mixed);
// FP32 inner solve of the mixed-precision path
void launch_apply0_32(Context& c, const float* x, float* y, const float* b);
void launch_dot32(Context& c, const float* a, const float* b, size_t n, double* out_dev);
void launch_axpy2_32(Context& c, const double* alpha_dev, const float* p, float* x, const float* q, float* r, size_t n);
void launch_xpby32(Context& c, const float* z, const double* beta_dev, float* p, size_t n);
void launch_zero_constrained32(Context& c, float* v);
void launch_vcycle32(Context& c, const float* r, float* z);
void autotune_vcycle32(Context& c);   // launch shapes of the FP32 V-cycle, once per hierarchy
void check_device_error(Context& c);  // raises when a bounded device wait ran out
void launch_d2f(Context& c, const double* a, float* b, size_t n);
void launch_add_f2d(Context& c, const float* d, double* x, size_t n);
void launch_f2d(Context& c, const float* a, double* b, size_t n);
void launch_div(Context& c, const double* num, const double* den, double* out, double sign);
void launch_scale_vec(Context& c, const double* x, const double* s, double* y, bool divide, size_t n);
void launch_finalize(Context& c, double* out_dev);                                  // sum of the last reduction partials
void launch_axpy(Context& c, double alpha, const double* x, double* y, size_t n);   // y += alpha x
void launch_div_scalar(Context& c, double* v, double d, size_t n);                  // v /= d

// ---- level-0 sweep of the FP32 V-cycle with TMA-streamed operator rows (tm_sweep_tma.cu)
void plan_sweep_tma(Context& c, const std::vector<int>* colPos, cudaStream_t st);
bool launch_sweep_tma(Context& c, int col, int zeroGuess, const float* b, float* x);   // false: not available
void launch_val_to_f32(Context& c);   // FP32 level-0 operator (and its position-major copy for the TMA sweep)
size_t sweep_tma_smem(int maxNodes, int nstage);   // shared memory of the TMA sweep (~0: does not fit)

// ---- matrix-free level 0 (tm_mf.cu) --------------------------------------------------------------
void mf_build_cells(Context& c, int stage);                 // cell classes for a stage (host, on a stage change)
void launch_mf_combine(Context& c);                         // combined cell matrices of the step (after the condensation)
void launch_mf_scales(Context& c, bool scaled);             // gs, os, cd of the unscaled or the scaled operator
void launch_mf_apply(Context& c, const double* x, double* y, const double* b);   // y = Ks x, or b - Ks x
void launch_mf_apply32(Context& c, const float* x, float* y, const float* b);
void launch_mf_sweep32(Context& c, int col, int zeroGuess, const float* b, float* x);   // one colour of the level-0 sweep
void launch_mf_sweep64(Context& c, int col, int zeroGuess, const double* b, double* x);
size_t mf_sweep_smem(int nz);

// ---- Anand (tm_anand.cu) ---------------------------------------------------------------------
void anand_screen_device(const tm_anand_material& mat, int nsites, int ntemps, const double* temps_h,
                         const double* table_d, int nsteps, const double* t_h, const double* T_h,
                         const int* cycle_h, const int* phase_h, int cycles, double* dW_d, double* dE_d,
                         double* stab_d, cudaStream_t s, const tm_pillar* pillar = nullptr, double* grad_d = nullptr);
void anand_step_device(const tm_anand_material& mat, int npts, double* state_d, const double* eps_d,
                       double T, double dt, double* sig_d, double* D_d, int commit, cudaStream_t s);

// ---- bump submodel (tm_submodel.cu) -------------------------------------------------------------
struct SubModel;
SubModel* submodel_create(const tm_submodel_spec& spec);
void submodel_destroy(SubModel* s);
bool submodel_step(SubModel& s, double T, double dt, int* newton, double* dMax);
void submodel_get(SubModel& s, double* u, double* W, double* ebar);
void submodel_sizes(SubModel& s, int64_t* out);
void submodel_run(SubModel& s, int nsteps, const double* t, const double* T, const int* cycle, int cycles, double cphi, double sphi,
                  double* out, double* perCycle, double* loop, const int* phase = nullptr, int maxSnaps = 0, int* nSnaps = nullptr,
                  double* snapMeta = nullptr, float* snapSig = nullptr);
void submodel_stress_snapshot(SubModel& s, double T, float* out);
void submodel_set_precond(SubModel& s, int kind);
void submodel_counters(SubModel& s, int64_t* out);
void submodel_run_batch(const std::vector<SubModel*>& subs, int nsteps, const double* t, const double* T, const int* cycle, int cycles,
                        const double* cphi, const double* sphi, double* out10, double* perCycle, double* loop, int32_t* status);

}  // namespace tmg
