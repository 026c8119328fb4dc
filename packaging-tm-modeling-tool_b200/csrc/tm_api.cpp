// C-ABI of the B200 solve path (include/tmsolve.h): context management, the PCG loop with
// the reference's warm start and rebuild policy, and the Anand entry points.
//
// The solve follows LinearSolver (src/core/10-solver.js:826-1043):
//   solve            :933-994   scaling, preconditioner (re)build, warm start, stale-preconditioner
//                               budget, rebuild on failure, rate bookkeeping, solution store
//   _pcg             :1001-1042 PCG on the scaled system with constrained DOFs zeroed in r and z
//   _warmStart       :885-915   Galerkin projection on <= 20 stored solutions
//   _storeSolution   :917-926   two-pass Gram-Schmidt
//   fallback         :967-976   after a failed rebuild, one more run with the other kind (MG <-> IC(0),
//                               ICPC on the device in tm_ic0.cu), then the preferred kind again
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <thread>
#include <chrono>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "tm_internal.h"

namespace tmg {

thread_local std::string g_last_error;

void set_last_error(const std::string& msg) { g_last_error = msg; }

void fail(tm_status st, const std::string& msg) { throw Error{st, msg}; }

void cuda_check(cudaError_t e, const char* what) {
  if (e != cudaSuccess) throw Error{TM_CUDA, std::string(what) + ": " + cudaGetErrorString(e)};
}

long long launch_count();

// the path has no CPU fallback: a usable sm_100 device or TM_NO_DEVICE
void require_device() {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) fail(TM_NO_DEVICE, "no CUDA device: the solve path has no CPU fallback");
  int dev = 0;
  TM_CUDA_CHECK(cudaGetDevice(&dev));
  cudaDeviceProp prop;
  TM_CUDA_CHECK(cudaGetDeviceProperties(&prop, dev));
  if (prop.major < 10) fail(TM_NO_DEVICE, std::string("device ") + prop.name + " is not sm_100: this library is built for B200 (sm_100a) only");
}

Context::~Context() {
  for (auto* L : shells) delete L;
  for (auto* b : basis) delete b;
  for (auto& e : timerEvents) { cudaEventDestroy(e.first); cudaEventDestroy(e.second); }
  for (auto& g : vcGraph) if (g) cudaGraphExecDestroy(g);
  if (capStream) cudaStreamDestroy(capStream);
  if (stream && ownStream) cudaStreamDestroy(stream);
}

namespace {

double now_ms() {
  using namespace std::chrono;
  return duration<double, std::milli>(steady_clock::now().time_since_epoch()).count();
}

template <class F>
tm_status guarded(F&& f) {
  try {
    f();
    return TM_OK;
  } catch (const Error& e) {
    g_last_error = e.msg;
    return e.status;
  } catch (const std::exception& e) {
    g_last_error = e.what();
    return TM_CUDA;
  }
}


// numeric set-up of a preconditioner for the current scaled operator (_buildPC, 10-solver.js:868-882):
// MultigridPC constructor / update, ICPC, or nothing for Jacobi (the scaled operator's diagonal is 1)
double build_pc(Context& c, int kind) {
  const double t0 = now_ms();
  c.pcKind = kind;
  if (kind == TM_PC_JACOBI) { c.pcReady = true; c.needRebuild = false; return now_ms() - t0; }
  if (kind == TM_PC_IC) {
    build_ic(c);
    c.pcReady = true;
    c.needRebuild = false;
    return now_ms() - t0;
  }
  c.d_jitter.zero(c.stream);
  {
    TimedLaunch tl(c, K_SETUP_LEVEL0);
    launch_factor_columns(c);
    launch_w01(c);
  }
  launch_galerkin01(c);
  for (size_t l = 0; l < c.shells.size(); l++) {
    ShellLevel& L = *c.shells[l];
    if (L.coarsest) {
      TimedLaunch tl(c, K_SETUP_COARSEST);
      launch_factor_coarsest(c, L);
      break;
    }
    TimedLaunch tl(c, K_SETUP_SHELL);
    launch_factor_shell(c, L);
    launch_galerkin_shell(c, (int)l);
  }
  int jit = 0;
  TM_CUDA_CHECK(cudaMemcpyAsync(&jit, c.d_jitter.p, sizeof(int), cudaMemcpyDeviceToHost, c.stream));
  TM_CUDA_CHECK(cudaStreamSynchronize(c.stream));
  c.colJitter = jit;
  c.pcReady = true;
  c.needRebuild = false;
  return now_ms() - t0;
}

void precondition(Context& c, int kind, const double* r, double* z) {
  const size_t n = 3 * (size_t)c.nn;
  const bool mg = kind == TM_PC_MG;
  if (kind == TM_PC_IC) launch_ic_apply(c, r, z);
  else if (mg && c.mgFp32) {
    // FP32 V-cycle (operators, column factors, transfers and smoothing in FP32; coarsest FP64)
    launch_d2f(c, r, c.d_r32.p, n);
    launch_vcycle32(c, c.d_r32.p, c.d_z32.p);
    launch_f2d(c, c.d_z32.p, z, n);
  } else if (mg) launch_vcycle(c, r, z, false);
  else TM_CUDA_CHECK(cudaMemcpyAsync(z, r, 3 * (size_t)c.nn * sizeof(double), cudaMemcpyDeviceToDevice, c.stream));
}

double dot_host(Context& c, const double* a, const double* b, size_t n) {
  launch_dot(c, a, b, n, c.d_scalars.p + 15);
  double v = 0;
  TM_CUDA_CHECK(cudaMemcpyAsync(&v, c.d_scalars.p + 15, sizeof(double), cudaMemcpyDeviceToHost, c.stream));
  TM_CUDA_CHECK(cudaStreamSynchronize(c.stream));
  return v;
}

struct PcgResult {
  int iters = 0;
  double relres = 0, iters0 = 0;
  bool converged = false;
  bool nonfinite = false;
};

// _pcg (10-solver.js:1001-1042); device scalars: 0 rz, 1 pq, 2 alpha, 3 r.r, 4 rz2, 5 beta
PcgResult pcg(Context& c, int kind, const double* b, double* x, double tol, int maxit, double perDecade, const tm_solve_opts& o) {
  const size_t n = 3 * (size_t)c.nn;
  double* S = c.d_scalars.p;
  PcgResult out;
  launch_apply0(c, x, c.d_r.p, b);
  launch_zero_constrained(c, c.d_r.p);
  launch_zero_constrained(c, x);
  const double bnorm = std::sqrt(dot_host(c, b, b, n));
  double rnorm = std::sqrt(dot_host(c, c.d_r.p, c.d_r.p, n));
  const double r0 = rnorm / bnorm;
  out.iters0 = r0;
  if (!std::isfinite(r0)) { out.nonfinite = true; out.relres = r0; return out; }
  if (rnorm / bnorm < tol) { out.iters = 0; out.relres = rnorm / bnorm; out.converged = true; return out; }
  if (perDecade > 0) maxit = std::min(maxit, std::max(30, (int)std::ceil(perDecade * std::log10(r0 / tol))));  // REBUILD_MIN_ITERS
  precondition(c, kind, c.d_r.p, c.d_z.p);
  launch_zero_constrained(c, c.d_z.p);
  TM_CUDA_CHECK(cudaMemcpyAsync(c.d_p.p, c.d_z.p, n * sizeof(double), cudaMemcpyDeviceToDevice, c.stream));
  launch_dot(c, c.d_r.p, c.d_z.p, n, S + 0);
  int it = 0;
  double hs[4];
  for (it = 1; it <= maxit; it++) {
    launch_apply0(c, c.d_p.p, c.d_q.p, nullptr);
    launch_dot(c, c.d_p.p, c.d_q.p, n, S + 1);
    launch_div(c, S + 0, S + 1, S + 2, 1.0);
    launch_axpy2(c, S + 2, c.d_p.p, x, c.d_q.p, c.d_r.p, n);
    launch_finalize(c, S + 3);   // r.r from the partial sums of k_axpy2
    TM_CUDA_CHECK(cudaMemcpyAsync(hs, S, 4 * sizeof(double), cudaMemcpyDeviceToHost, c.stream));
    TM_CUDA_CHECK(cudaStreamSynchronize(c.stream));
    const double pq = hs[1];
    if (!(pq > 0)) {
      // the reference breaks before the update; undo it (x -= alpha p, r += alpha q)
      double na = -hs[2];
      TM_CUDA_CHECK(cudaMemcpyAsync(S + 2, &na, sizeof(double), cudaMemcpyHostToDevice, c.stream));
      launch_axpy2(c, S + 2, c.d_p.p, x, c.d_q.p, c.d_r.p, n);
      if (!std::isfinite(pq)) out.nonfinite = true;
      break;
    }
    rnorm = std::sqrt(hs[3]);
    if (!std::isfinite(rnorm)) { out.nonfinite = true; break; }
    if (o.progress && o.progress_every > 0 && it % o.progress_every == 0) o.progress(o.progress_user, it, rnorm / bnorm);
    if (rnorm / bnorm < tol) { out.iters = it; out.relres = rnorm / bnorm; out.converged = true; return out; }
    precondition(c, kind, c.d_r.p, c.d_z.p);
    launch_zero_constrained(c, c.d_z.p);
    launch_dot(c, c.d_r.p, c.d_z.p, n, S + 4);
    launch_div(c, S + 4, S + 0, S + 5, 1.0);
    TM_CUDA_CHECK(cudaMemcpyAsync(S + 0, S + 4, sizeof(double), cudaMemcpyDeviceToDevice, c.stream));
    launch_xpby(c, c.d_z.p, S + 5, c.d_p.p, n);
  }
  out.iters = std::min(it, maxit);
  out.relres = rnorm / bnorm;
  out.converged = false;
  return out;
}

// Gauss-Jordan solve of the small warm-start system (solveDense / invDense, 01-util.js:110-142)
bool solve_dense(const std::vector<double>& A, int n, const std::vector<double>& b, std::vector<double>& x) {
  const int w = 2 * n;
  std::vector<double> M((size_t)n * w, 0.0);
  for (int i = 0; i < n; i++) {
    for (int j = 0; j < n; j++) M[i * w + j] = A[i * n + j];
    M[i * w + n + i] = 1;
  }
  for (int col = 0; col < n; col++) {
    int p = col;
    double best = std::fabs(M[col * w + col]);
    for (int r = col + 1; r < n; r++) { const double v = std::fabs(M[r * w + col]); if (v > best) { best = v; p = r; } }
    if (best == 0) return false;
    if (p != col) for (int j = 0; j < w; j++) std::swap(M[col * w + j], M[p * w + j]);
    const double inv = 1 / M[col * w + col];
    for (int j = 0; j < w; j++) M[col * w + j] *= inv;
    for (int r = 0; r < n; r++) {
      if (r == col) continue;
      const double f = M[r * w + col];
      if (f == 0) continue;
      for (int j = 0; j < w; j++) M[r * w + j] -= f * M[col * w + j];
    }
  }
  x.assign(n, 0.0);
  for (int i = 0; i < n; i++) {
    double s = 0;
    for (int j = 0; j < n; j++) s += M[i * w + n + j] * b[j];
    x[i] = s;
  }
  return true;
}

// _warmStart (10-solver.js:885-915) on the device
void warm_start(Context& c, const double* fs, double* x) {
  const size_t n = 3 * (size_t)c.nn;
  const int m = (int)c.basis.size();
  TM_CUDA_CHECK(cudaMemsetAsync(x, 0, n * sizeof(double), c.stream));
  if (!m) return;
  if (c.d_warmKV.n < (size_t)m * n) c.d_warmKV.alloc((size_t)m * n);
  std::vector<const double*> V(m), W(m + 1);
  for (int i = 0; i < m; i++) {
    double* kv = c.d_warmKV.p + (size_t)i * n;
    launch_scale_vec(c, c.basis[i]->p, c.d_s.p, c.d_tmp.p, true, n);
    launch_apply0(c, c.d_tmp.p, c.d_tmp2.p, nullptr);
    launch_scale_vec(c, c.d_tmp2.p, c.d_s.p, kv, true, n);
    V[i] = c.basis[i]->p;
    W[i] = kv;
  }
  launch_scale_vec(c, fs, c.d_s.p, c.d_tmp.p, true, n);
  W[m] = c.d_tmp.p;
  // A[i][j] = v_i . K v_j and b[i] = v_i . f: one batched launch, every dot independent as in the
  // reference's loops
  std::vector<double> AB((size_t)m * (m + 1)), A((size_t)m * m), b(m), cc;
  multi_dot_host(c, V, W, n, AB.data());
  for (int i = 0; i < m; i++) {
    for (int j = 0; j < m; j++) A[i * m + j] = AB[(size_t)i * (m + 1) + j];
    b[i] = AB[(size_t)i * (m + 1) + m];
  }
  for (int i = 0; i < m; i++)
    for (int j = i + 1; j < m; j++) { const double v = 0.5 * (A[i * m + j] + A[j * m + i]); A[i * m + j] = A[j * m + i] = v; }
  if (!solve_dense(A, m, b, cc)) return;
  for (int i = 0; i < m; i++) if (!std::isfinite(cc[i])) return;
  for (int i = 0; i < m; i++) launch_axpy(c, cc[i], c.basis[i]->p, x, n);
  launch_scale_vec(c, x, c.d_s.p, x, true, n);
}

// _storeSolution (10-solver.js:917-926)
void store_solution(Context& c, const double* u_dev, int warmMax) {
  if (warmMax <= 0) return;
  const size_t n = 3 * (size_t)c.nn;
  auto* v = new DBuf<double>();
  v->alloc(n);
  TM_CUDA_CHECK(cudaMemcpyAsync(v->p, u_dev, n * sizeof(double), cudaMemcpyDeviceToDevice, c.stream));
  for (int pass = 0; pass < 2; pass++)
    for (auto* b : c.basis) launch_axpy(c, -dot_host(c, b->p, v->p, n), b->p, v->p, n);
  const double nv = std::sqrt(dot_host(c, v->p, v->p, n));
  const double nu = std::sqrt(dot_host(c, u_dev, u_dev, n));
  if (!(nv > 1e-14 * (nu + 1e-300))) { delete v; return; }
  launch_div_scalar(c, v->p, nv, n);
  c.basis.push_back(v);
  while ((int)c.basis.size() > warmMax) { delete c.basis.front(); c.basis.erase(c.basis.begin()); }
}

// FP32 PCG on K d = r32 from d = 0 (inner solve of the mixed-precision refinement): the
// stiffness apply and the V-cycle run in FP32 with FP32 accumulation; dots accumulate in FP64.
PcgResult pcg32(Context& c, double tol_in, int maxit) {
  const size_t n = 3 * (size_t)c.nn;
  double* S = c.d_scalars.p;
  PcgResult out;
  TM_CUDA_CHECK(cudaMemsetAsync(c.d_d32.p, 0, n * sizeof(float), c.stream));
  const double r0n = std::sqrt([&] {
    launch_dot32(c, c.d_r32.p, c.d_r32.p, n, S + 15);
    double v = 0;
    TM_CUDA_CHECK(cudaMemcpyAsync(&v, S + 15, sizeof(double), cudaMemcpyDeviceToHost, c.stream));
    TM_CUDA_CHECK(cudaStreamSynchronize(c.stream));
    return v;
  }());
  if (!(r0n > 0)) { out.converged = true; return out; }
  launch_vcycle32(c, c.d_r32.p, c.d_z32.p);
  launch_zero_constrained32(c, c.d_z32.p);
  TM_CUDA_CHECK(cudaMemcpyAsync(c.d_p32.p, c.d_z32.p, n * sizeof(float), cudaMemcpyDeviceToDevice, c.stream));
  launch_dot32(c, c.d_r32.p, c.d_z32.p, n, S + 0);
  int it = 0;
  double hs[4];
  for (it = 1; it <= maxit; it++) {
    launch_apply0_32(c, c.d_p32.p, c.d_q32.p, nullptr);
    launch_dot32(c, c.d_p32.p, c.d_q32.p, n, S + 1);
    launch_div(c, S + 0, S + 1, S + 2, 1.0);
    launch_axpy2_32(c, S + 2, c.d_p32.p, c.d_d32.p, c.d_q32.p, c.d_r32.p, n);
    launch_finalize(c, S + 3);
    TM_CUDA_CHECK(cudaMemcpyAsync(hs, S, 4 * sizeof(double), cudaMemcpyDeviceToHost, c.stream));
    TM_CUDA_CHECK(cudaStreamSynchronize(c.stream));
    if (!(hs[1] > 0)) {
      double na = -hs[2];
      TM_CUDA_CHECK(cudaMemcpyAsync(S + 2, &na, sizeof(double), cudaMemcpyHostToDevice, c.stream));
      launch_axpy2_32(c, S + 2, c.d_p32.p, c.d_d32.p, c.d_q32.p, c.d_r32.p, n);
      if (!std::isfinite(hs[1])) out.nonfinite = true;
      break;
    }
    const double rn = std::sqrt(hs[3]);
    if (!std::isfinite(rn)) { out.nonfinite = true; break; }
    out.relres = rn / r0n;
    if (rn < tol_in * r0n) { out.iters = it; out.converged = true; return out; }
    launch_vcycle32(c, c.d_r32.p, c.d_z32.p);
    launch_zero_constrained32(c, c.d_z32.p);
    launch_dot32(c, c.d_r32.p, c.d_z32.p, n, S + 4);
    launch_div(c, S + 4, S + 0, S + 5, 1.0);
    TM_CUDA_CHECK(cudaMemcpyAsync(S + 0, S + 4, sizeof(double), cudaMemcpyDeviceToDevice, c.stream));
    launch_xpby32(c, c.d_z32.p, S + 5, c.d_p32.p, n);
  }
  out.iters = std::min(it, maxit);
  return out;
}

// TM_PREC_MIXED_IR: FP64 iterative refinement around an FP32 multigrid-PCG. Every sweep
// recomputes the FP64 residual r = b - K x, solves K d = r in FP32 (FP32 apply and V-cycle) to a
// relative 1e-4 and adds d to x in FP64. When a sweep fails to halve the FP64 residual (the
// FP32 operator's rounding times the condition number reaches 1, as on finely meshed lidded
// packages) *stalled is set and the caller continues with FP64 PCG and the FP32 V-cycle.
PcgResult refine_mixed(Context& c, const double* b, double* x, double tol, int maxit, int* sweeps, bool* stalled, const tm_solve_opts& o) {
  const size_t n = 3 * (size_t)c.nn;
  PcgResult out;
  launch_zero_constrained(c, x);
  const double bnorm = std::sqrt(dot_host(c, b, b, n));
  int total = 0;
  *sweeps = 0;
  *stalled = false;
  double prev = 0;
  for (int guard = 0; guard < 50; guard++) {
    launch_apply0(c, x, c.d_r.p, b);
    launch_zero_constrained(c, c.d_r.p);
    const double rel = std::sqrt(dot_host(c, c.d_r.p, c.d_r.p, n)) / bnorm;
    if (guard == 0) out.iters0 = rel;
    out.relres = rel;
    if (!std::isfinite(rel)) { out.nonfinite = true; break; }
    if (rel < tol) { out.converged = true; break; }
    if (guard > 0 && rel > 0.5 * prev) { *stalled = true; break; }
    prev = rel;
    if (total >= maxit) break;
    launch_d2f(c, c.d_r.p, c.d_r32.p, n);
    const double tol_in = std::max(1e-4, 0.3 * tol / rel);
    PcgResult in = pcg32(c, tol_in, maxit - total);
    total += in.iters;
    if (in.nonfinite) { out.nonfinite = true; break; }
    launch_add_f2d(c, c.d_d32.p, x, n);
    (*sweeps)++;
    if (o.progress && o.progress_every > 0) o.progress(o.progress_user, total, rel);
  }
  out.iters = total;
  return out;
}

double pcg_rate(const PcgResult& r) { return r.iters / std::max(std::log10(r.iters0 / std::max(r.relres, 1e-300)), 0.5); }

// LinearSolver.solve (10-solver.js:933-994) with f and u in device memory
tm_status solve_impl(Context& c, const double* f_dev, double* u_dev, const tm_solve_opts& o, tm_solve_info* info) {
  const double t0 = now_ms();
  if (!c.assembled) fail(TM_BAD_INPUT, "tm_solve before tm_assemble_step or tm_set_bcsr");
  const size_t n = 3 * (size_t)c.nn;
  if (o.precond != TM_PC_MG && o.precond != TM_PC_JACOBI && o.precond != TM_PC_IC) fail(TM_BAD_INPUT, "unknown preconditioner kind");
  const int kind = o.precond;
  const bool mg = kind == TM_PC_MG;
  if (o.key != -1 && o.key != c.pcKey) c.needRebuild = true;
  if (c.pcKind != kind) c.needRebuild = true;
  c.pcKey = o.key;
  if (!c.scaled) {
    launch_scale(c);
    launch_mf_scales(c, true);
    c.scaled = true;
    c.fp32Ready = false;
  }
  launch_scale_rhs(c, f_dev, c.d_bs.p);
  const double bnorm = std::sqrt(dot_host(c, c.d_bs.p, c.d_bs.p, n));
  tm_solve_info in;
  std::memset(&in, 0, sizeof(in));
  in.levels = mg ? (int)c.shells.size() + 1 : 1;
  if (!std::isfinite(bnorm)) fail(TM_NONFINITE, "non-finite load vector");
  if (bnorm == 0) {
    TM_CUDA_CHECK(cudaMemsetAsync(u_dev, 0, n * sizeof(double), c.stream));
    TM_CUDA_CHECK(cudaStreamSynchronize(c.stream));
    in.converged = 1; in.ms = now_ms() - t0; in.warm = (int)c.basis.size();
    if (info) *info = in;
    return TM_OK;
  }
  bool rebuilt = false;
  double pcMs = 0;
  const bool mixed = o.precision == TM_PREC_MIXED || o.precision == TM_PREC_MIXED_IR;
  if (mixed && !mg) fail(TM_BAD_INPUT, "mixed precision needs the multigrid preconditioner");
  c.mgFp32 = false;
  if (!c.pcReady || c.needRebuild) {
    pcMs = build_pc(c, kind);
    rebuilt = true;
    if (mixed) {
      const double t1 = now_ms();
      {
        TimedLaunch tl(c, K_TO_FP32);
        launch_to_fp32(c);
      }
      autotune_vcycle32(c);
      TM_CUDA_CHECK(cudaStreamSynchronize(c.stream));
      pcMs += now_ms() - t1;
      c.fp32Ready = true;
    }
  } else if (mixed && !c.fp32Ready) {
    launch_to_fp32(c);
    autotune_vcycle32(c);
    c.fp32Ready = true;
  }
  warm_start(c, c.d_bs.p, c.d_x.p);
  int sweeps = 0;
  bool stalled = false;
  PcgResult res;
  int total = 0;
  if (o.precision == TM_PREC_MIXED_IR) {
    res = refine_mixed(c, c.d_bs.p, c.d_x.p, o.tol, o.maxit, &sweeps, &stalled, o);
    if (stalled && !res.nonfinite) {
      c.mgFp32 = true;
      PcgResult r2 = pcg(c, kind, c.d_bs.p, c.d_x.p, o.tol, std::max(1, o.maxit - res.iters), 0, o);
      r2.iters += res.iters;
      r2.iters0 = res.iters0;
      res = r2;
    }
    total = res.iters;
  } else {
    c.mgFp32 = o.precision == TM_PREC_MIXED;
    res = pcg(c, kind, c.d_bs.p, c.d_x.p, o.tol, o.maxit, rebuilt ? 0 : 2 * c.ratePerDecade, o);   // REBUILD_FACTOR 2
    total = res.iters;
    if (!res.converged && !rebuilt && !res.nonfinite) {
      // stale preconditioner: rebuild the preferred kind and continue from the current iterate
      pcMs += build_pc(c, kind);
      rebuilt = true;
      res = pcg(c, kind, c.d_bs.p, c.d_x.p, o.tol, o.maxit, 0, o);
      total += res.iters;
    }
  }
  bool fellBack = false;
  if (!res.converged && !res.nonfinite) {
    // rebuild with the other kind once, keeping the current iterate (FP64 PCG), then return to the
    // preferred kind on the next solve
    const int first = c.pcKind, other = first == TM_PC_MG ? TM_PC_IC : TM_PC_MG;
    in.fallback = 1;
    in.fallback_first = first;
    in.fallback_iters = total;
    in.fallback_relres = res.relres;
    pcMs += build_pc(c, other);
    rebuilt = true;
    c.mgFp32 = false;
    res = pcg(c, other, c.d_bs.p, c.d_x.p, o.tol, o.maxit, 0, o);
    total += res.iters;
    c.needRebuild = true;
    fellBack = true;
  }
  if (!res.converged) c.needRebuild = true;
  if (res.converged && !fellBack) {
    const bool known = c.ratePerDecade > 0 && !rebuilt;
    if (known) { if (pcg_rate(res) > 2 * c.ratePerDecade) c.needRebuild = true; }
    else c.ratePerDecade = std::log10(res.iters0 / std::max(res.relres, 1e-300)) >= 1 ? pcg_rate(res) : 0;
  }
  // u = x * s
  launch_scale_vec(c, c.d_x.p, c.d_s.p, u_dev, false, n);
  TM_CUDA_CHECK(cudaStreamSynchronize(c.stream));
  if (res.converged) store_solution(c, u_dev, o.warm);
  in.iters = total; in.relres = res.relres; in.iters0 = res.iters0; in.converged = res.converged;
  in.ms = now_ms() - t0; in.pc_ms = pcMs; in.rebuilt = rebuilt; in.warm = (int)c.basis.size();
  in.jitter_count = c.colJitter; in.refinements = sweeps;
  in.precond = c.pcKind;
  check_device_error(c);
  in.status = res.nonfinite ? TM_NONFINITE : (res.converged ? TM_OK : TM_NOT_CONVERGED);
  if (info) *info = in;
  if (res.nonfinite) fail(TM_NONFINITE, "non-finite value in the PCG iteration");
  return res.converged ? TM_OK : TM_NOT_CONVERGED;
}

void upload_mesh(Context& c) {
  cudaStream_t s = c.stream;
  {
    c.nnp = (c.nn + 3) / 4 * 4;
    std::vector<int> pn((size_t)NSLOT * c.nnp, -1);
    for (int sl = 0; sl < NSLOT; sl++)
      for (int n = 0; n < c.nn; n++) pn[(size_t)sl * c.nnp + c.pos[n]] = c.nbr[(size_t)sl * c.nn + n];
    c.d_nbr.upload(pn, s);
  }
  c.d_pos.upload(c.pos, s);
  c.d_posNode.upload(c.posNode, s);
  c.d_slotMask.upload(c.slotMask, s);
  c.d_nodeIJK.upload(c.nodeIJK, s);
  c.d_cellElems.upload(c.cellElems, s);
  c.d_eGroup.upload(c.eGroup, s);
  c.d_groupStage.upload(c.groupStage, s);
  c.d_eClass.upload(c.eClass, s);
  c.d_colStart.upload(c.colStart, s);
  c.d_eScale.upload(c.eScale, s);
  c.d_clsPset.upload(c.clsPset, s);
  c.d_clsH.upload(c.clsH, s);
  c.d_constr.upload(c.constr, s);
  const size_t n = 3 * (size_t)c.nn;
  for (auto* b : {&c.d_f, &c.d_bs, &c.d_x, &c.d_r, &c.d_z, &c.d_p, &c.d_q, &c.d_tmp, &c.d_tmp2}) b->alloc(n);
  c.d_partial.alloc(1024);
  c.d_scalars.alloc(16);
  c.d_jitter.alloc(1);
  c.d_err.alloc(1);
  c.d_err.zero(s);
}

}  // namespace

// a bounded device wait that ran out (the results of the solve are invalid)
void check_device_error(Context& c) {
  int err = 0;
  TM_CUDA_CHECK(cudaMemcpyAsync(&err, c.d_err.p, sizeof(int), cudaMemcpyDeviceToHost, c.stream));
  TM_CUDA_CHECK(cudaStreamSynchronize(c.stream));
  if (err) {
    c.d_err.zero(c.stream);
    TM_CUDA_CHECK(cudaStreamSynchronize(c.stream));
    fail(TM_TIMEOUT, "a bounded wait of the level-0 sweep ran out");
  }
}

}  // namespace tmg

using namespace tmg;

extern "C" {

void tm_default_solve_opts(tm_solve_opts* o) {
  std::memset(o, 0, sizeof(*o));
  o->tol = 1e-8;
  o->maxit = 2000;
  o->warm = 20;
  o->precond = TM_PC_MG;
  o->precision = TM_PREC_FP64;
  o->key = -1;
}

int32_t tm_last_error(char* buf, size_t len) {
  if (buf && len) {
    const size_t k = std::min(len - 1, g_last_error.size());
    std::memcpy(buf, g_last_error.data(), k);
    buf[k] = 0;
  }
  return (int32_t)g_last_error.size();
}

tm_status tm_create(const tm_mesh* m, tm_ctx** out) {
  return guarded([&] {
    if (!m || !out) fail(TM_BAD_INPUT, "null argument");
    *out = nullptr;
    require_device();
    if (m->nx < 2 || m->ny < 2 || m->nz < 2 || m->nn <= 0 || m->ne <= 0) fail(TM_BAD_INPUT, "empty mesh");
    auto* c = new Context();
    try {
      TM_CUDA_CHECK(cudaGetDevice(&c->dev));
      TM_CUDA_CHECK(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
      c->nx = m->nx; c->ny = m->ny; c->nz = m->nz; c->nn = m->nn; c->ne = m->ne; c->npset = m->npset; c->ngroups = m->ngroups;
      const size_t ncells = (size_t)(m->nx - 1) * (m->ny - 1) * (m->nz - 1);
      c->xs.assign(m->xs, m->xs + m->nx); c->ys.assign(m->ys, m->ys + m->ny); c->zs.assign(m->zs, m->zs + m->nz);
      c->coords.assign(m->coords, m->coords + 3 * (size_t)m->nn);
      c->nodeId.assign(m->nodeId, m->nodeId + (size_t)m->nx * m->ny * m->nz);
      c->conn.assign(m->conn, m->conn + 8 * (size_t)m->ne);
      c->eIJK.assign(m->eIJK, m->eIJK + 3 * (size_t)m->ne);
      c->colStart.assign(m->colStart, m->colStart + (size_t)m->nx * m->ny + 1);
      c->cellElems.assign(m->cellElems, m->cellElems + 2 * ncells);
      c->eGroup.assign(m->eGroup, m->eGroup + m->ne);
      c->ePart.assign(m->ePart, m->ePart + m->ne);
      c->eScale.assign(m->eScale, m->eScale + m->ne);
      c->groupStage.assign(m->groupStage, m->groupStage + m->ngroups);
      c->ePset.assign(m->ePset, m->ePset + m->ne);
      c->constr.assign(m->constr, m->constr + m->nconstr);
      if (m->nfeatureX > 0) c->featureX.assign(m->featureX, m->featureX + m->nfeatureX);
      if (m->nfeatureY > 0) c->featureY.assign(m->featureY, m->featureY + m->nfeatureY);
      c->meshConstr = c->constr;
      if (m->nmodconstr > 0) {   // the model's module constraints: the package's then the modules' (09-assembly.js:227)
        if (!m->modconstr) fail(TM_BAD_INPUT, "module constraints: null list");
        c->modConstr = c->constr;
        c->modConstr.insert(c->modConstr.end(), m->modconstr, m->modconstr + m->nmodconstr);
      }
      // index validation (no device access is made with unchecked indices)
      for (int v : c->conn) if (v < 0 || v >= c->nn) fail(TM_BAD_INPUT, "conn index out of range");
      for (int v : c->nodeId) if (v >= c->nn) fail(TM_BAD_INPUT, "nodeId out of range");
      for (int v : c->cellElems) if (v >= c->ne) fail(TM_BAD_INPUT, "cellElems out of range");
      for (int v : c->eGroup) if (v < 0 || v >= c->ngroups) fail(TM_BAD_INPUT, "eGroup out of range");
      for (int v : c->ePset) if (v < 0 || v >= c->npset) fail(TM_BAD_INPUT, "ePset out of range");
      for (int v : c->constr) if (v < 0 || v >= 3 * c->nn) fail(TM_BAD_INPUT, "constraint DOF out of range");
      for (int v : c->modConstr) if (v < 0 || v >= 3 * c->nn) fail(TM_BAD_INPUT, "module constraint DOF out of range");
      if (c->colStart.back() != c->nn) fail(TM_BAD_INPUT, "colStart does not cover the nodes");
      build_stencil(*c);
      build_classes(*c);
      upload_mesh(*c);
      build_hierarchy(*c);
      TM_CUDA_CHECK(cudaStreamSynchronize(c->stream));
    } catch (...) {
      delete c;
      throw;
    }
    *out = reinterpret_cast<tm_ctx*>(c);
  });
}

tm_status tm_destroy(tm_ctx* ctx) {
  return guarded([&] { delete reinterpret_cast<Context*>(ctx); });
}

namespace {
void check_step(const Context& c, const tm_step& st) {
  for (int p = 0; p < c.npset; p++) {
    const double* src = st.psetLayered[p] ? st.W + 108 * (size_t)p : st.D + 36 * (size_t)p;
    const int cnt = st.psetLayered[p] ? 108 : 36;
    for (int q = 0; q < cnt; q++) if (!std::isfinite(src[q])) fail(TM_NONFINITE, "non-finite property-set stiffness");
  }
}
}  // namespace

namespace {
// the active set and constraints of a stage (moduleStageSet / moduleStageConstraints,
// 09-assembly.js:427-443): in a stacked-module stage the born elements, the nodes they touch and
// the module constraints plus every DOF of the other nodes (sorted); otherwise the whole package
// with the mesh's constraints. A change of the active set rebuilds the hierarchy (the reference's
// _buildPC keyed on activeKey, 10-solver.js:868-876).
void set_active_stage(Context& c, int stage) {
  const bool moduleStage = stage < 0 && !c.modConstr.empty();
  c.moduleStage = moduleStage;
  const int key = moduleStage ? stage : 0;
  if (moduleStage) {
    c.actElem.assign(c.ne, 0);
    c.actNode.assign(c.nn, 0);
    for (int e = 0; e < c.ne; e++) {
      if (c.groupStage[c.eGroup[e]] > stage) continue;
      c.actElem[e] = 1;
      for (int a = 0; a < 8; a++) c.actNode[c.conn[8 * (size_t)e + a]] = 1;
    }
    std::vector<uint8_t> fixed(3 * (size_t)c.nn, 0);
    for (int d : c.modConstr) fixed[d] = 1;
    for (int n = 0; n < c.nn; n++)
      if (!c.actNode[n]) fixed[3 * (size_t)n] = fixed[3 * (size_t)n + 1] = fixed[3 * (size_t)n + 2] = 1;
    c.constr.clear();
    for (int d = 0; d < 3 * c.nn; d++) if (fixed[d]) c.constr.push_back(d);
  } else {
    c.actElem.clear();
    c.actNode.clear();
    c.constr = c.meshConstr;   // (a caller-assembled operator, tm_set_bcsr, may have loaded its own list)
  }
  c.d_constr.upload(c.constr, c.stream);
  if (key != c.hierKey) {
    c.activeKey = key;
    build_hierarchy(c);
    c.hierKey = key;
    c.needRebuild = true;
    c.pcReady = false;
  }
}
}  // namespace

tm_status tm_prepare_step(tm_ctx* ctx, const tm_step* st) {
  return guarded([&] {
    if (!ctx || !st) fail(TM_BAD_INPUT, "null argument");
    Context& c = *reinterpret_cast<Context*>(ctx);
    check_step(c, *st);
    launch_shape_matrices(c, *st);
    TM_CUDA_CHECK(cudaStreamSynchronize(c.stream));
  });
}

tm_status tm_assemble_step(tm_ctx* ctx, const tm_step* st, double* rhs_out) {
  return guarded([&] {
    if (!ctx || !st) fail(TM_BAD_INPUT, "null argument");
    Context& c = *reinterpret_cast<Context*>(ctx);
    check_step(c, *st);
    launch_shape_matrices(c, *st);
    launch_class_condense(c);
    set_active_stage(c, st->stage);
    if (c.level0Mf) {
      mf_build_cells(c, st->stage);
      launch_mf_combine(c);
    }
    launch_assemble(c);
    launch_constraints(c);
    c.assembled = true;
    c.scaled = false;
    c.mf = c.level0Mf && c.mfAvailable;
    launch_mf_scales(c, false);
    if (rhs_out) {
      c.d_rhs.download(rhs_out, 3 * (size_t)c.nn, c.stream);
    }
    TM_CUDA_CHECK(cudaStreamSynchronize(c.stream));
  });
}

tm_status tm_assemble_step_device(tm_ctx* ctx, const tm_step* st, double* rhs_dev) {
  tm_status s = tm_assemble_step(ctx, st, nullptr);
  if (s != TM_OK || !rhs_dev) return s;
  return guarded([&] {
    Context& c = *reinterpret_cast<Context*>(ctx);
    TM_CUDA_CHECK(cudaMemcpyAsync(rhs_dev, c.d_rhs.p, 3 * (size_t)c.nn * sizeof(double), cudaMemcpyDeviceToDevice, c.stream));
    TM_CUDA_CHECK(cudaStreamSynchronize(c.stream));
  });
}

tm_status tm_set_bcsr(tm_ctx* ctx, const int32_t* rowPtr, const int32_t* col, const double* val, const uint8_t* isConstrained) {
  return guarded([&] {
    Context& c = *reinterpret_cast<Context*>(ctx);
    const int nn = c.nn, S = c.nnp;
    std::vector<double> sv((size_t)NSLOT * 9 * S, 0.0);
    for (int i = 0; i < nn; i++) {
      const int ii = c.nodeIJK[3 * (size_t)i], ij = c.nodeIJK[3 * (size_t)i + 1], ik = c.nodeIJK[3 * (size_t)i + 2];
      for (int k = rowPtr[i]; k < rowPtr[i + 1]; k++) {
        const int j = col[k];
        if (j < 0 || j >= nn) fail(TM_BAD_INPUT, "block column out of range");
        const int di = c.nodeIJK[3 * (size_t)j] - ii, dj = c.nodeIJK[3 * (size_t)j + 1] - ij, dk = c.nodeIJK[3 * (size_t)j + 2] - ik;
        if (std::abs(di) > 1 || std::abs(dj) > 1 || std::abs(dk) > 1) fail(TM_BAD_INPUT, "block outside the 27-point stencil of the mesh");
        const int s = (di + 1) * 9 + (dj + 1) * 3 + (dk + 1);
        for (int v = 0; v < 9; v++) sv[((size_t)s * 9 + v) * S + c.pos[i]] = val[9 * (size_t)k + v];
      }
    }
    c.d_val.upload(sv, c.stream);
    c.constr.clear();
    for (int d = 0; d < 3 * nn; d++) if (isConstrained && isConstrained[d]) c.constr.push_back(d);
    c.d_constr.upload(c.constr, c.stream);
    c.assembled = true;
    c.scaled = false;
    c.mf = false;   // a caller-assembled operator has no element classes: the stencil path
    TM_CUDA_CHECK(cudaStreamSynchronize(c.stream));
  });
}

tm_status tm_get_bcsr(tm_ctx* ctx, int32_t* rowPtr, int32_t* col, double* val) {
  return guarded([&] {
    Context& c = *reinterpret_cast<Context*>(ctx);
    const int nn = c.nn, S = c.nnp;
    std::vector<double> sv((size_t)NSLOT * 9 * S);
    c.d_val.download(sv.data(), sv.size(), c.stream);
    TM_CUDA_CHECK(cudaStreamSynchronize(c.stream));
    int k = 0;
    if (rowPtr) rowPtr[0] = 0;
    for (int i = 0; i < nn; i++) {
      for (int s = 0; s < NSLOT; s++) {
        if (!(c.slotMask[i] >> s & 1)) continue;
        if (col) col[k] = c.nbr[(size_t)s * nn + i];
        if (val) for (int v = 0; v < 9; v++) val[9 * (size_t)k + v] = sv[((size_t)s * 9 + v) * S + c.pos[i]];
        k++;
      }
      if (rowPtr) rowPtr[i + 1] = k;
    }
  });
}

tm_status tm_sizes(tm_ctx* ctx, int64_t* out) {
  return guarded([&] {
    Context& c = *reinterpret_cast<Context*>(ctx);
    long long nb = 0;
    for (int i = 0; i < c.nn; i++) nb += __builtin_popcount((unsigned)c.slotMask[i]);
    out[0] = c.nn; out[1] = c.ne; out[2] = nb; out[3] = 3LL * c.nn;
    out[4] = (int64_t)c.shells.size() + 1;
    out[5] = c.shells.empty() ? 0 : c.shells.back()->denseN;
  });
}

tm_status tm_matvec_device(tm_ctx* ctx, const double* x, double* y) {
  return guarded([&] {
    Context& c = *reinterpret_cast<Context*>(ctx);
    if (!c.assembled) fail(TM_BAD_INPUT, "tm_matvec before an operator is loaded");
    launch_apply0(c, x, y, nullptr);
    TM_CUDA_CHECK(cudaStreamSynchronize(c.stream));
  });
}

tm_status tm_matvec(tm_ctx* ctx, const double* x, double* y) {
  return guarded([&] {
    Context& c = *reinterpret_cast<Context*>(ctx);
    if (!c.assembled) fail(TM_BAD_INPUT, "tm_matvec before an operator is loaded");
    const size_t n = 3 * (size_t)c.nn;
    c.d_tmp.upload(x, n, c.stream);
    launch_apply0(c, c.d_tmp.p, c.d_tmp2.p, nullptr);
    c.d_tmp2.download(y, n, c.stream);
    TM_CUDA_CHECK(cudaStreamSynchronize(c.stream));
  });
}

// ---- element DOF histories (Model.accumulateStep qOnly) and strains at points -------------------
namespace {
void recovery_ready(Context& c) {
  if (!c.stepReady) fail(TM_BAD_INPUT, "element DOF histories need a step loaded by tm_prepare_step or tm_assemble_step");
  if (!c.d_conn.p) c.d_conn.upload(c.conn, c.stream);
}
void check_elems(const Context& c, int32_t n, const int32_t* e) {
  for (int32_t t = 0; t < n; t++)
    if (e[t] >= c.ne) fail(TM_BAD_INPUT, "element index out of range");
}
}  // namespace

tm_status tm_accumulate_q_device(tm_ctx* ctx, const double* du, int32_t nel, const int32_t* elems, double* q) {
  return guarded([&] {
    Context& c = *reinterpret_cast<Context*>(ctx);
    if (nel < 0 || (nel > 0 && (!du || !elems || !q))) fail(TM_BAD_INPUT, "tm_accumulate_q: bad arguments");
    recovery_ready(c);
    launch_accumulate_q(c, du, nel, elems, q);
    TM_CUDA_CHECK(cudaStreamSynchronize(c.stream));
  });
}

tm_status tm_accumulate_q(tm_ctx* ctx, const double* du, int32_t nel, const int32_t* elems, double* q) {
  return guarded([&] {
    Context& c = *reinterpret_cast<Context*>(ctx);
    if (nel < 0 || (nel > 0 && (!du || !elems || !q))) fail(TM_BAD_INPUT, "tm_accumulate_q: bad arguments");
    if (nel == 0) return;
    check_elems(c, nel, elems);
    recovery_ready(c);
    DBuf<int> de;
    DBuf<double> dq;
    c.d_tmp.upload(du, 3 * (size_t)c.nn, c.stream);
    de.upload(elems, nel, c.stream);
    dq.upload(q, 33 * (size_t)nel, c.stream);
    launch_accumulate_q(c, c.d_tmp.p, nel, de.p, dq.p);
    dq.download(q, 33 * (size_t)nel, c.stream);
    TM_CUDA_CHECK(cudaStreamSynchronize(c.stream));
  });
}

// ---- element stress histories (Model.accumulateStep without qOnly, stateStress) ---------------------
tm_status tm_set_sublayers(tm_ctx* ctx, const int32_t* nsub, const double* subZ, const double* subD, const double* subS0) {
  return guarded([&] {
    Context& c = *reinterpret_cast<Context*>(ctx);
    if (!nsub) fail(TM_BAD_INPUT, "tm_set_sublayers: null argument");
    if (!c.stepReady) fail(TM_BAD_INPUT, "tm_set_sublayers after tm_prepare_step or tm_assemble_step");
    std::vector<int> off(c.npset + 1, 0);
    int mx = 1;
    for (int p = 0; p < c.npset; p++) {
      if (nsub[p] < 0) fail(TM_BAD_INPUT, "tm_set_sublayers: negative sub-layer count");
      off[p + 1] = off[p] + nsub[p];
      mx = std::max(mx, (int)nsub[p]);
    }
    std::vector<int> lay(c.npset);
    TM_CUDA_CHECK(cudaMemcpyAsync(lay.data(), c.d_psetLayered.p, c.npset * sizeof(int), cudaMemcpyDeviceToHost, c.stream));
    TM_CUDA_CHECK(cudaStreamSynchronize(c.stream));
    for (int p = 0; p < c.npset; p++)
      if (lay[p] && nsub[p] < 1) fail(TM_BAD_INPUT, "tm_set_sublayers: a layered property set needs its sub-layers");
    const size_t n = off[c.npset];
    if (n && (!subZ || !subD || !subS0)) fail(TM_BAD_INPUT, "tm_set_sublayers: null sub-layer data");
    c.d_subOff.upload(off, c.stream);
    if (n) {
      c.d_subZ.upload(subZ, 2 * n, c.stream); c.d_subD.upload(subD, 36 * n, c.stream); c.d_subS0.upload(subS0, 6 * n, c.stream);
    } else {
      c.d_subZ.alloc(2); c.d_subD.alloc(36); c.d_subS0.alloc(6);
    }
    c.maxSub = mx;
    c.subReady = true;
    TM_CUDA_CHECK(cudaStreamSynchronize(c.stream));
  });
}

namespace {
void state_ready(Context& c, int32_t stride) {
  recovery_ready(c);
  if (!c.subReady) fail(TM_BAD_INPUT, "stress histories need the step's sub-layers (tm_set_sublayers)");
  if (stride < 33 + 48 * c.maxSub) fail(TM_BAD_INPUT, "state stride below 33 + 48 x the largest sub-layer count");
  if (!c.d_eIJK.p) { c.d_eIJK.upload(c.eIJK, c.stream); c.d_zs.upload(c.zs, c.stream); }
}
}  // namespace

tm_status tm_accumulate_state_device(tm_ctx* ctx, const double* du, int32_t nel, const int32_t* elems, int32_t stride, double* state) {
  return guarded([&] {
    Context& c = *reinterpret_cast<Context*>(ctx);
    if (nel < 0 || (nel > 0 && (!du || !elems || !state))) fail(TM_BAD_INPUT, "tm_accumulate_state: bad arguments");
    state_ready(c, stride);
    launch_accumulate_state(c, du, nel, elems, stride, state);
    TM_CUDA_CHECK(cudaStreamSynchronize(c.stream));
  });
}

tm_status tm_accumulate_state(tm_ctx* ctx, const double* du, int32_t nel, const int32_t* elems, int32_t stride, double* state) {
  return guarded([&] {
    Context& c = *reinterpret_cast<Context*>(ctx);
    if (nel < 0 || (nel > 0 && (!du || !elems || !state))) fail(TM_BAD_INPUT, "tm_accumulate_state: bad arguments");
    if (nel == 0) return;
    check_elems(c, nel, elems);
    state_ready(c, stride);
    DBuf<int> de;
    DBuf<double> ds;
    c.d_tmp.upload(du, 3 * (size_t)c.nn, c.stream);
    de.upload(elems, nel, c.stream);
    ds.upload(state, (size_t)stride * nel, c.stream);
    launch_accumulate_state(c, c.d_tmp.p, nel, de.p, stride, ds.p);
    ds.download(state, (size_t)stride * nel, c.stream);
    TM_CUDA_CHECK(cudaStreamSynchronize(c.stream));
  });
}

tm_status tm_state_stress_device(tm_ctx* ctx, int32_t npts, const int32_t* elem, const double* state, int32_t stride, const double* nat,
                                 double* eps, double* sig) {
  return guarded([&] {
    Context& c = *reinterpret_cast<Context*>(ctx);
    if (npts < 0 || (npts > 0 && (!elem || !state || !nat || !eps || !sig))) fail(TM_BAD_INPUT, "tm_state_stress: bad arguments");
    state_ready(c, stride);
    launch_state_stress(c, npts, elem, state, stride, nat, eps, sig);
    TM_CUDA_CHECK(cudaStreamSynchronize(c.stream));
  });
}

tm_status tm_state_stress(tm_ctx* ctx, int32_t npts, const int32_t* elem, const double* state, int32_t stride, const double* nat,
                          double* eps, double* sig) {
  return guarded([&] {
    Context& c = *reinterpret_cast<Context*>(ctx);
    if (npts < 0 || (npts > 0 && (!elem || !state || !nat || !eps || !sig))) fail(TM_BAD_INPUT, "tm_state_stress: bad arguments");
    if (npts == 0) return;
    check_elems(c, npts, elem);
    state_ready(c, stride);
    DBuf<int> de;
    DBuf<double> ds, dn, de6, ds6;
    de.upload(elem, npts, c.stream);
    ds.upload(state, (size_t)stride * npts, c.stream);
    dn.upload(nat, 3 * (size_t)npts, c.stream);
    de6.alloc(6 * (size_t)npts); ds6.alloc(6 * (size_t)npts);
    launch_state_stress(c, npts, de.p, ds.p, stride, dn.p, de6.p, ds6.p);
    de6.download(eps, 6 * (size_t)npts, c.stream);
    ds6.download(sig, 6 * (size_t)npts, c.stream);
    TM_CUDA_CHECK(cudaStreamSynchronize(c.stream));
  });
}

tm_status tm_element_strains_device(tm_ctx* ctx, int32_t npts, const int32_t* elem, const double* q, const double* nat, double* eps) {
  return guarded([&] {
    Context& c = *reinterpret_cast<Context*>(ctx);
    if (npts < 0 || (npts > 0 && (!elem || !q || !nat || !eps))) fail(TM_BAD_INPUT, "tm_element_strains: bad arguments");
    launch_element_strains(c, npts, elem, q, nat, eps);
    TM_CUDA_CHECK(cudaStreamSynchronize(c.stream));
  });
}

tm_status tm_element_strains(tm_ctx* ctx, int32_t npts, const int32_t* elem, const double* q, const double* nat, double* eps) {
  return guarded([&] {
    Context& c = *reinterpret_cast<Context*>(ctx);
    if (npts < 0 || (npts > 0 && (!elem || !q || !nat || !eps))) fail(TM_BAD_INPUT, "tm_element_strains: bad arguments");
    if (npts == 0) return;
    check_elems(c, npts, elem);
    DBuf<int> de;
    DBuf<double> dq, dn, deps;
    de.upload(elem, npts, c.stream);
    dq.upload(q, 33 * (size_t)npts, c.stream);
    dn.upload(nat, 3 * (size_t)npts, c.stream);
    deps.alloc(6 * (size_t)npts);
    launch_element_strains(c, npts, de.p, dq.p, dn.p, deps.p);
    deps.download(eps, 6 * (size_t)npts, c.stream);
    TM_CUDA_CHECK(cudaStreamSynchronize(c.stream));
  });
}

// ---- the transposes of the strain recovery, for adjoints of functions of the site strains --------------
tm_status tm_element_strains_adjoint(tm_ctx* ctx, int32_t npts, const int32_t* elem, const double* nat, const double* g, double* gq) {
  return guarded([&] {
    Context& c = *reinterpret_cast<Context*>(ctx);
    if (npts < 0 || (npts > 0 && (!elem || !nat || !g || !gq))) fail(TM_BAD_INPUT, "tm_element_strains_adjoint: bad arguments");
    if (npts == 0) return;
    check_elems(c, npts, elem);
    DBuf<int> de;
    DBuf<double> dn, dg, dgq;
    de.upload(elem, npts, c.stream);
    dn.upload(nat, 3 * (size_t)npts, c.stream);
    dg.upload(g, 6 * (size_t)npts, c.stream);
    dgq.alloc(33 * (size_t)npts);
    launch_element_strains_adjoint(c, npts, de.p, dn.p, dg.p, dgq.p);
    dgq.download(gq, 33 * (size_t)npts, c.stream);
    TM_CUDA_CHECK(cudaStreamSynchronize(c.stream));
  });
}

tm_status tm_accumulate_q_adjoint(tm_ctx* ctx, int32_t nel, const int32_t* elems, const double* gq, double* gdu, double* gA) {
  return guarded([&] {
    Context& c = *reinterpret_cast<Context*>(ctx);
    if (nel < 0 || (nel > 0 && (!elems || !gq || !gdu || !gA))) fail(TM_BAD_INPUT, "tm_accumulate_q_adjoint: bad arguments");
    if (nel == 0) return;
    check_elems(c, nel, elems);
    recovery_ready(c);
    DBuf<int> de;
    DBuf<double> dgq, dgdu, dgA;
    de.upload(elems, nel, c.stream);
    dgq.upload(gq, 33 * (size_t)nel, c.stream);
    dgdu.alloc(24 * (size_t)nel);
    dgA.alloc(nel);
    launch_accumulate_q_adjoint(c, nel, de.p, dgq.p, dgdu.p, dgA.p);
    dgdu.download(gdu, 24 * (size_t)nel, c.stream);
    dgA.download(gA, nel, c.stream);
    TM_CUDA_CHECK(cudaStreamSynchronize(c.stream));
  });
}

// ---- samplePlane at points ------------------------------------------------------------------------
tm_status tm_sample_plane_device(tm_ctx* ctx, const double* u, int32_t k, int32_t comp, int32_t npts, const double* x,
                                 const double* y, double* out) {
  return guarded([&] {
    Context& c = *reinterpret_cast<Context*>(ctx);
    if (k < 0 || k >= c.nz || comp < 0 || comp > 2 || npts < 0 || (npts > 0 && (!u || !x || !y || !out)))
      fail(TM_BAD_INPUT, "tm_sample_plane: bad arguments");
    launch_sample_plane(c, u, k, comp, npts, x, y, out);
    TM_CUDA_CHECK(cudaStreamSynchronize(c.stream));
  });
}

tm_status tm_sample_plane(tm_ctx* ctx, const double* u, int32_t k, int32_t comp, int32_t npts, const double* x, const double* y,
                          double* out) {
  return guarded([&] {
    Context& c = *reinterpret_cast<Context*>(ctx);
    if (k < 0 || k >= c.nz || comp < 0 || comp > 2 || npts < 0 || (npts > 0 && (!u || !x || !y || !out)))
      fail(TM_BAD_INPUT, "tm_sample_plane: bad arguments");
    if (npts == 0) return;
    DBuf<double> dx, dy, dout;
    c.d_tmp.upload(u, 3 * (size_t)c.nn, c.stream);
    dx.upload(x, npts, c.stream);
    dy.upload(y, npts, c.stream);
    dout.alloc(npts);
    launch_sample_plane(c, c.d_tmp.p, k, comp, npts, dx.p, dy.p, dout.p);
    dout.download(out, npts, c.stream);
    TM_CUDA_CHECK(cudaStreamSynchronize(c.stream));
  });
}

tm_status tm_pc_apply_device(tm_ctx* ctx, const double* r, double* z) {
  return guarded([&] {
    Context& c = *reinterpret_cast<Context*>(ctx);
    if (!c.pcReady || c.pcKind < 0) fail(TM_BAD_INPUT, "tm_pc_apply before a solve built a preconditioner");
    c.mgFp32 = false;
    precondition(c, c.pcKind, r, z);
    TM_CUDA_CHECK(cudaStreamSynchronize(c.stream));
  });
}

tm_status tm_set_vcycle_shapes(tm_ctx* ctx, int nlevels, const int* wpb_sweep, const int* wpb_apply, int tma_stages) {
  return guarded([&] {
    Context& c = *reinterpret_cast<Context*>(ctx);
    auto okw = [](int w) { return w == 2 || w == 4 || w == 8; };
    if (nlevels < 0) {
      c.shapesPinned = false;
    } else {
      if (nlevels > 0 && (!wpb_sweep || !wpb_apply)) fail(TM_BAD_INPUT, "tm_set_vcycle_shapes: missing per-level arrays");
      if (tma_stages != 0 && tma_stages != 2 && tma_stages != 3) fail(TM_BAD_INPUT, "tm_set_vcycle_shapes: TMA stages must be 0, 2 or 3");
      for (int k = 0; k < nlevels; k++)
        if (!okw(wpb_sweep[k]) || !okw(wpb_apply[k])) fail(TM_BAD_INPUT, "tm_set_vcycle_shapes: warps per block must be 2, 4 or 8");
      c.pinSweep.assign(wpb_sweep, wpb_sweep + nlevels);
      c.pinApply.assign(wpb_apply, wpb_apply + nlevels);
      c.pinStages = tma_stages;
      c.shapesPinned = true;
    }
    c.tunedEpoch = -1;   // applied (or tuned again) before the next FP32 V-cycle
  });
}

tm_status tm_vcycle_shapes(tm_ctx* ctx, int cap, int* nlevels, int* wpb_sweep, int* wpb_apply, int* tma_stages) {
  return guarded([&] {
    Context& c = *reinterpret_cast<Context*>(ctx);
    if (c.tunedEpoch != c.structEpoch) fail(TM_BAD_INPUT, "tm_vcycle_shapes before a mixed-precision solve tuned the V-cycle");
    int k = 0;
    for (auto* L : c.shells) {
      if (L->coarsest || !L->colorCount[0]) continue;
      if (k < cap) {
        if (wpb_sweep) wpb_sweep[k] = L->wpbSweep;
        if (wpb_apply) wpb_apply[k] = L->wpbApply;
      }
      k++;
    }
    if (nlevels) *nlevels = k;
    if (tma_stages) *tma_stages = c.tsReady && !c.mf ? c.tsStages : 0;
  });
}

tm_status tm_mg_levels(tm_ctx* ctx, int32_t cap, int32_t* out4, int32_t* nlevels) {
  return guarded([&] {
    if (!ctx) fail(TM_BAD_INPUT, "null context");
    Context& c = *reinterpret_cast<Context*>(ctx);
    if (!c.hierarchy) fail(TM_BAD_INPUT, "no multigrid hierarchy");
    const int L = 1 + (int)c.shells.size();
    if (nlevels) *nlevels = L;
    if (!out4) return;
    for (int l = 0; l < L && l < cap; l++) {
      int32_t* o = out4 + 4 * l;
      if (l == 0) { o[0] = c.nx; o[1] = c.ny; o[2] = c.nn; o[3] = 3; }
      else { const ShellLevel& S = *c.shells[l - 1]; o[0] = S.nx; o[1] = S.ny; o[2] = S.nn; o[3] = 6; }
    }
  });
}

tm_status tm_shell_sweep_bytes(tm_ctx* ctx, double* bytes_per_cycle, int32_t* launches_per_cycle) {
  return guarded([&] {
    if (!ctx) fail(TM_BAD_INPUT, "null context");
    Context& c = *reinterpret_cast<Context*>(ctx);
    if (!c.hierarchy) fail(TM_BAD_INPUT, "no multigrid hierarchy");
    double bytes = 0;
    int launches = 0;
    for (const ShellLevel* Lp : c.shells) {
      const ShellLevel& L = *Lp;
      if (L.coarsest) break;
      const double f = sizeof(float), ncol = (double)L.nx * L.ny;
      const double inverses = f * (L.cfPtr.empty() ? 0.0 : (double)L.cfPtr.back());
      const double vec = f * 6.0 * L.nn;          // one level vector
      const double lists = 24.0 * ncol;           // per column: aggregate/block ranges, inverse offset
      const double full = (36.0 * f + 4.0) * L.nb + inverses + 3.0 * vec + lists;   // b, x read, x write
      // the cycle's first launch on the level (the first non-empty colour, i = j = 0 mod 2 when
      // present) starts from x = 0 and reads neither the blocks nor x of its columns
      int k0 = 0;
      while (k0 < 4 && !L.colorCount[k0]) k0++;
      double blk0 = 0, agg0 = 0;
      for (int cc = 0; cc < L.nx * L.ny; cc++) {
        const int i = cc / L.ny, j = cc % L.ny;
        if ((i & 1) * 2 + (j & 1) != k0) continue;
        blk0 += L.rowPtr[L.colStart[cc + 1]] - L.rowPtr[L.colStart[cc]];
        agg0 += L.colStart[cc + 1] - L.colStart[cc];
      }
      bytes += 4.0 * full - (36.0 * f + 4.0) * blk0 - f * 6.0 * agg0;
      int colours = 0;
      for (int k = 0; k < 4; k++) colours += L.colorCount[k] ? 1 : 0;
      launches += 4 * colours;
    }
    if (bytes_per_cycle) *bytes_per_cycle = bytes;
    if (launches_per_cycle) *launches_per_cycle = launches;
  });
}

tm_status tm_mg_node_agg(tm_ctx* ctx, int32_t* out) {
  return guarded([&] {
    if (!ctx || !out) fail(TM_BAD_INPUT, "null argument");
    Context& c = *reinterpret_cast<Context*>(ctx);
    if (!c.hierarchy) fail(TM_BAD_INPUT, "no multigrid hierarchy");
    std::copy(c.nodeAgg.begin(), c.nodeAgg.end(), out);
  });
}

tm_status tm_set_wait_test(tm_ctx* ctx, int32_t on) {
  return guarded([&] {
    if (!ctx) fail(TM_BAD_INPUT, "null context");
    reinterpret_cast<Context*>(ctx)->waitTest = on != 0;
  });
}

tm_status tm_clear_warm(tm_ctx* ctx) {
  return guarded([&] {
    if (!ctx) fail(TM_BAD_INPUT, "null context");
    Context& c = *reinterpret_cast<Context*>(ctx);
    TM_CUDA_CHECK(cudaStreamSynchronize(c.stream));
    for (auto* b : c.basis) delete b;
    c.basis.clear();
  });
}

tm_status tm_set_level0(tm_ctx* ctx, int32_t matrix_free) {
  return guarded([&] {
    if (!ctx) fail(TM_BAD_INPUT, "null context");
    reinterpret_cast<Context*>(ctx)->level0Mf = matrix_free != 0;
  });
}

tm_status tm_level0(tm_ctx* ctx, int32_t* matrix_free_active) {
  return guarded([&] {
    if (!ctx || !matrix_free_active) fail(TM_BAD_INPUT, "null argument");
    *matrix_free_active = reinterpret_cast<Context*>(ctx)->mf ? 1 : 0;
  });
}

tm_status tm_pc_apply(tm_ctx* ctx, const double* r, double* z) {
  return guarded([&] {
    Context& c = *reinterpret_cast<Context*>(ctx);
    if (!c.pcReady || c.pcKind < 0) fail(TM_BAD_INPUT, "tm_pc_apply before a solve built a preconditioner");
    const size_t n = 3 * (size_t)c.nn;
    c.mgFp32 = false;
    c.d_tmp.upload(r, n, c.stream);
    c.d_tmp2.alloc(n);
    precondition(c, c.pcKind, c.d_tmp.p, c.d_tmp2.p);
    c.d_tmp2.download(z, n, c.stream);
    TM_CUDA_CHECK(cudaStreamSynchronize(c.stream));
  });
}

tm_status tm_solve_device(tm_ctx* ctx, const double* f_dev, double* u_dev, const tm_solve_opts* opts, tm_solve_info* info) {
  tm_status st = TM_OK;
  tm_status g = guarded([&] {
    Context& c = *reinterpret_cast<Context*>(ctx);
    tm_solve_opts o;
    if (opts) o = *opts; else tm_default_solve_opts(&o);
    st = solve_impl(c, f_dev, u_dev, o, info);
  });
  return g != TM_OK ? g : st;
}

tm_status tm_solve(tm_ctx* ctx, const double* f, double* u, const tm_solve_opts* opts, tm_solve_info* info) {
  tm_status st = TM_OK;
  tm_status g = guarded([&] {
    Context& c = *reinterpret_cast<Context*>(ctx);
    const size_t n = 3 * (size_t)c.nn;
    tm_solve_opts o;
    if (opts) o = *opts; else tm_default_solve_opts(&o);
    // the load's finiteness is checked on the device (its scaled norm); the staging buffers
    // persist across calls, so a solve allocates nothing after the first
    c.d_f.upload(f, n, c.stream);
    c.d_uio.alloc(n);
    st = solve_impl(c, c.d_f.p, c.d_uio.p, o, info);
    c.d_uio.download(u, n, c.stream);
    TM_CUDA_CHECK(cudaStreamSynchronize(c.stream));
  });
  return g != TM_OK ? g : st;
}

// tm_solve with the displacement returned as float32, rounded on the device (the solution kept
// for post-processing and the results file is Float32, 11-analysis.js:256)
tm_status tm_solve_f32(tm_ctx* ctx, const double* f, float* u32, const tm_solve_opts* opts, tm_solve_info* info) {
  tm_status st = TM_OK;
  tm_status g = guarded([&] {
    Context& c = *reinterpret_cast<Context*>(ctx);
    if (!f || !u32) fail(TM_BAD_INPUT, "null argument");
    const size_t n = 3 * (size_t)c.nn;
    tm_solve_opts o;
    if (opts) o = *opts; else tm_default_solve_opts(&o);
    c.d_f.upload(f, n, c.stream);
    c.d_uio.alloc(n);
    st = solve_impl(c, c.d_f.p, c.d_uio.p, o, info);
    c.d_u32out.alloc(n);
    launch_d2f(c, c.d_uio.p, c.d_u32out.p, n);
    c.d_u32out.download(u32, n, c.stream);
    TM_CUDA_CHECK(cudaStreamSynchronize(c.stream));
  });
  return g != TM_OK ? g : st;
}

// adjoint sensitivities of the smooth warpage measure J = mean over the nodes of plane k of the
// squared residual of their z displacement about its least-squares plane (fitPlane,
// 01-util.js:176-190): dJ/du = 2 r / N on those z DOFs; K lambda = dJ/du by the same solver
// (free DOFs); per property set m, with K_m and f_m the set's share of the assembled operator and
// load, dJ/dlog(E_m) = lambda^T (f_m - K_m u) (K_m and f_m scale with the set's stiffness) and
// dJ/dlog(alpha_m) = lambda^T f_m (f_m scales with its thermal strain)
namespace {
// the adjoint solve K lambda = g (no warm start, nothing stored; constrained DOFs of g zeroed) and,
// per property set m with K_m and f_m its share of the step's operator and load, dlogE_m =
// lambda^T (f_m - K_m u) and dlogA_m = lambda^T f_m, summed per element on the device
tm_status adjoint_sums(Context& c, const double* g, const double* u, const tm_solve_opts* opts, double* dlogE, double* dlogA,
                       tm_solve_info* info) {
  const size_t n = 3 * (size_t)c.nn;
  tm_solve_opts o;
  if (opts) o = *opts; else tm_default_solve_opts(&o);
  o.warm = 0;
  c.d_f.upload(g, n, c.stream);
  launch_zero_constrained(c, c.d_f.p);
  c.d_sensLam.alloc(n);
  const tm_status st = solve_impl(c, c.d_f.p, c.d_sensLam.p, o, info);
  c.d_sensU.upload(u, n, c.stream);
  if (!c.d_conn.p) c.d_conn.upload(c.conn, c.stream);
  std::vector<double> sums(2 * (size_t)c.npset);
  launch_sens(c, c.d_sensU.p, c.d_sensLam.p, sums.data());
  for (int p = 0; p < c.npset; p++) { dlogE[p] = sums[2 * p + 1] - sums[2 * p]; dlogA[p] = sums[2 * p + 1]; }
  c.sensReady = true;
  return st;
}
}  // namespace

tm_status tm_warpage_sensitivity(tm_ctx* ctx, const double* u, int32_t k, const tm_solve_opts* opts, double* J, double* dlogE,
                                 double* dlogA, tm_solve_info* info) {
  tm_status st = TM_OK;
  tm_status g = guarded([&] {
    Context& c = *reinterpret_cast<Context*>(ctx);
    if (!u || !J || !dlogE || !dlogA) fail(TM_BAD_INPUT, "null argument");
    if (!c.assembled || !c.stepReady || !c.d_clsKc.p) fail(TM_BAD_INPUT, "sensitivities need a step assembled by tm_assemble_step");
    if (k < 0 || k >= c.nz) fail(TM_BAD_INPUT, "plane index out of range");
    const size_t n = 3 * (size_t)c.nn;
    // the plane's nodes, the fitted plane and the measure's gradient
    std::vector<int> nodes;
    for (int q = 0; q < c.nn; q++) if (c.nodeIJK[3 * (size_t)q + 2] == k) nodes.push_back(q);
    const int N = (int)nodes.size();
    if (N < 3) fail(TM_BAD_INPUT, "plane with fewer than 3 nodes");
    double sx = 0, sy = 0, sw = 0;
    for (int q : nodes) { sx += c.xs[c.nodeIJK[3 * (size_t)q]]; sy += c.ys[c.nodeIJK[3 * (size_t)q + 1]]; sw += u[3 * (size_t)q + 2]; }
    const double mx = sx / N, my = sy / N, mw = sw / N;
    double sxx = 0, sxy = 0, syy = 0, sxw = 0, syw = 0;
    for (int q : nodes) {
      const double dx = c.xs[c.nodeIJK[3 * (size_t)q]] - mx, dy = c.ys[c.nodeIJK[3 * (size_t)q + 1]] - my, dw = u[3 * (size_t)q + 2] - mw;
      sxx += dx * dx; sxy += dx * dy; syy += dy * dy; sxw += dx * dw; syw += dy * dw;
    }
    const double det = sxx * syy - sxy * sxy;
    double c1 = 0, c2 = 0;
    if (std::fabs(det) > 1e-300) { c1 = (sxw * syy - syw * sxy) / det; c2 = (syw * sxx - sxw * sxy) / det; }
    const double c0 = mw - c1 * mx - c2 * my;
    std::vector<double> gr(n, 0.0);
    double Jv = 0;
    for (int q : nodes) {
      const double r = u[3 * (size_t)q + 2] - (c0 + c1 * c.xs[c.nodeIJK[3 * (size_t)q]] + c2 * c.ys[c.nodeIJK[3 * (size_t)q + 1]]);
      Jv += r * r;
      gr[3 * (size_t)q + 2] = 2 * r / N;
    }
    *J = Jv / N;
    st = adjoint_sums(c, gr.data(), u, opts, dlogE, dlogA, info);
  });
  return g != TM_OK ? g : st;
}

tm_status tm_adjoint_sensitivity(tm_ctx* ctx, const double* g, const double* u, const tm_solve_opts* opts, double* dlogE, double* dlogA,
                                 tm_solve_info* info) {
  tm_status st = TM_OK;
  tm_status gs = guarded([&] {
    Context& c = *reinterpret_cast<Context*>(ctx);
    if (!g || !u || !dlogE || !dlogA) fail(TM_BAD_INPUT, "null argument");
    if (!c.assembled || !c.stepReady || !c.d_clsKc.p) fail(TM_BAD_INPUT, "sensitivities need a step assembled by tm_assemble_step");
    for (size_t q = 0; q < 3 * (size_t)c.nn; q++) if (!std::isfinite(g[q])) fail(TM_NONFINITE, "non-finite adjoint load");
    st = adjoint_sums(c, g, u, opts, dlogE, dlogA, info);
  });
  return gs != TM_OK ? gs : st;
}

tm_status tm_sensitivity_direction(tm_ctx* ctx, const tm_step* base, const tm_step* dir, double* dJ) {
  return guarded([&] {
    Context& c = *reinterpret_cast<Context*>(ctx);
    if (!base || !dir || !dJ) fail(TM_BAD_INPUT, "null argument");
    if (!c.sensReady) fail(TM_BAD_INPUT, "tm_sensitivity_direction after tm_warpage_sensitivity");
    check_step(c, *base);
    sens_direction(c, *base, *dir, c.d_sensU.p, c.d_sensLam.p, dJ);
  });
}

tm_status tm_set_stream(tm_ctx* ctx, void* stream) {
  return guarded([&] {
    Context& c = *reinterpret_cast<Context*>(ctx);
    TM_CUDA_CHECK(cudaStreamSynchronize(c.stream));
    if (c.ownStream && c.stream) cudaStreamDestroy(c.stream);
    c.stream = reinterpret_cast<cudaStream_t>(stream);
    c.ownStream = false;
  });
}

int64_t tm_launch_count(void) { return (int64_t)launch_count(); }

tm_status tm_kernel_timer(tm_ctx* ctx, int32_t kernel) {
  return guarded([&] {
    Context& c = *reinterpret_cast<Context*>(ctx);
    if (kernel < -1 || kernel >= K_NKERNEL) fail(TM_BAD_INPUT, "unknown kernel id");
    TM_CUDA_CHECK(cudaStreamSynchronize(c.stream));
    for (auto& e : c.timerEvents) { cudaEventDestroy(e.first); cudaEventDestroy(e.second); }
    c.timerEvents.clear();
    c.timerKernel = kernel;
  });
}

tm_status tm_kernel_timer_read(tm_ctx* ctx, int64_t* count, double* total_ms) {
  return guarded([&] {
    Context& c = *reinterpret_cast<Context*>(ctx);
    TM_CUDA_CHECK(cudaStreamSynchronize(c.stream));
    double tot = 0;
    for (auto& e : c.timerEvents) {
      float ms = 0;
      TM_CUDA_CHECK(cudaEventElapsedTime(&ms, e.first, e.second));
      tot += ms;
      cudaEventDestroy(e.first);
      cudaEventDestroy(e.second);
    }
    *count = (int64_t)c.timerEvents.size();
    *total_ms = tot;
    c.timerEvents.clear();
  });
}

tm_status tm_anand_screen_device(const tm_anand_material* mat, int32_t nsites, int32_t ntemps, const double* temps, const double* table_dev,
                                 int32_t nsteps, const double* t, const double* T, const int32_t* cycle, const int32_t* phase, int32_t cycles,
                                 double* dW, double* dE, double* stab) {
  return guarded([&] {
    require_device();
    anand_screen_device(*mat, nsites, ntemps, temps, table_dev, nsteps, t, T, cycle, phase, cycles, dW, dE, stab, nullptr);
  });
}

tm_status tm_anand_screen(const tm_anand_material* mat, int32_t nsites, int32_t ntemps, const double* temps, const double* table,
                          int32_t nsteps, const double* t, const double* T, const int32_t* cycle, const int32_t* phase, int32_t cycles,
                          double* dW, double* dE, double* stab) {
  return guarded([&] {
    require_device();
    if (nsites <= 0) return;
    DBuf<double> d_tab, d_dW, d_dE, d_st;
    d_tab.upload(table, (size_t)nsites * ntemps * 6, nullptr);
    d_dW.alloc(nsites); d_dE.alloc(nsites); d_st.alloc(nsites);
    anand_screen_device(*mat, nsites, ntemps, temps, d_tab.p, nsteps, t, T, cycle, phase, cycles, d_dW.p, d_dE.p, d_st.p, nullptr);
    d_dW.download(dW, nsites, nullptr); d_dE.download(dE, nsites, nullptr); d_st.download(stab, nsites, nullptr);
    TM_CUDA_CHECK(cudaDeviceSynchronize());
  });
}

tm_status tm_anand_screen_pillar_device(const tm_anand_material* mat, const tm_pillar* pillar, int32_t nsites, int32_t ntemps,
                                        const double* temps, const double* table_dev, int32_t nsteps, const double* t, const double* T,
                                        const int32_t* cycle, const int32_t* phase, int32_t cycles, double* dW, double* dE,
                                        double* stab) {
  return guarded([&] {
    require_device();
    if (!mat || !pillar) fail(TM_BAD_INPUT, "null argument");
    if (nsites <= 0) return;
    anand_screen_device(*mat, nsites, ntemps, temps, table_dev, nsteps, t, T, cycle, phase, cycles, dW, dE, stab, nullptr, pillar);
  });
}

tm_status tm_anand_screen_pillar(const tm_anand_material* mat, const tm_pillar* pillar, int32_t nsites, int32_t ntemps,
                                 const double* temps, const double* table, int32_t nsteps, const double* t, const double* T,
                                 const int32_t* cycle, const int32_t* phase, int32_t cycles, double* dW, double* dE, double* stab) {
  return guarded([&] {
    require_device();
    if (!mat || !pillar) fail(TM_BAD_INPUT, "null argument");
    if (nsites <= 0) return;
    DBuf<double> d_tab, d_dW, d_dE, d_st;
    d_tab.upload(table, (size_t)nsites * ntemps * 6, nullptr);
    d_dW.alloc(nsites); d_dE.alloc(nsites); d_st.alloc(nsites);
    anand_screen_device(*mat, nsites, ntemps, temps, d_tab.p, nsteps, t, T, cycle, phase, cycles, d_dW.p, d_dE.p, d_st.p, nullptr,
                        pillar);
    d_dW.download(dW, nsites, nullptr); d_dE.download(dE, nsites, nullptr); d_st.download(stab, nsites, nullptr);
    TM_CUDA_CHECK(cudaDeviceSynchronize());
  });
}

tm_status tm_anand_screen_gradient(const tm_anand_material* mat, const tm_pillar* pillar, int32_t ntemps, const double* temps,
                                   const double* table, int32_t nsteps, const double* t, const double* T, const int32_t* cycle,
                                   const int32_t* phase, int32_t cycles, double* dW, double* dE, double* gW, double* gE) {
  return guarded([&] {
    if (!mat || !temps || !table || !t || !T || !cycle || !phase || !dW || !dE || !gW || !gE) fail(TM_BAD_INPUT, "null argument");
    require_device();
    const size_t nt = 6 * (size_t)ntemps;
    for (size_t i = 0; i < nt; i++) if (!std::isfinite(table[i])) fail(TM_NONFINITE, "the site's strain table has a non-finite entry");
    cudaStream_t s = nullptr;
    TM_CUDA_CHECK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    try {
      DBuf<double> d_tab, d_out;
      d_tab.upload(table, nt, s);
      d_out.alloc(2 + 2 * nt);
      anand_screen_device(*mat, 1, ntemps, temps, d_tab.p, nsteps, t, T, cycle, phase, cycles, nullptr, nullptr, nullptr, s, pillar, d_out.p);
      std::vector<double> h(2 + 2 * nt);
      d_out.download(h.data(), h.size(), s);
      TM_CUDA_CHECK(cudaStreamSynchronize(s));
      *dW = h[0]; *dE = h[1];
      std::copy(h.begin() + 2, h.begin() + 2 + nt, gW);
      std::copy(h.begin() + 2 + nt, h.end(), gE);
    } catch (...) {
      cudaStreamDestroy(s);
      throw;
    }
    cudaStreamDestroy(s);
  });
}

tm_status tm_anand_step(const tm_anand_material* mat, int32_t npts, double* state, const double* eps, double T, double dt, double* sig,
                        double* D, int32_t commit) {
  return guarded([&] {
    require_device();
    if (npts <= 0) return;
    DBuf<double> d_state, d_eps, d_sig, d_D;
    d_state.upload(state, 12 * (size_t)npts, nullptr);
    d_eps.upload(eps, 6 * (size_t)npts, nullptr);
    d_sig.alloc(6 * (size_t)npts);
    if (D) d_D.alloc(36 * (size_t)npts);
    anand_step_device(*mat, npts, d_state.p, d_eps.p, T, dt, d_sig.p, D ? d_D.p : nullptr, commit, nullptr);
    d_state.download(state, 12 * (size_t)npts, nullptr);
    d_sig.download(sig, 6 * (size_t)npts, nullptr);
    if (D) d_D.download(D, 36 * (size_t)npts, nullptr);
    TM_CUDA_CHECK(cudaDeviceSynchronize());
  });
}

// ---- bump submodel ----------------------------------------------------------------------------------
tm_status tm_submodel_create(const tm_submodel_spec* spec, tm_sub** out) {
  return guarded([&] {
    require_device();
    if (!spec || !out) fail(TM_BAD_INPUT, "null argument");
    *out = reinterpret_cast<tm_sub*>(submodel_create(*spec));
  });
}

tm_status tm_submodel_set_precond(tm_sub* sm, int32_t kind) {
  return guarded([&] {
    if (!sm) fail(TM_BAD_INPUT, "null argument");
    submodel_set_precond(*reinterpret_cast<SubModel*>(sm), kind);
  });
}

tm_status tm_submodel_counters(tm_sub* sm, int64_t* out2) {
  return guarded([&] {
    if (!sm || !out2) fail(TM_BAD_INPUT, "null argument");
    submodel_counters(*reinterpret_cast<SubModel*>(sm), out2);
  });
}

tm_status tm_submodel_destroy(tm_sub* sm) {
  return guarded([&] { submodel_destroy(reinterpret_cast<SubModel*>(sm)); });
}

tm_status tm_submodel_sizes(tm_sub* sm, int64_t* out) {
  return guarded([&] {
    if (!sm || !out) fail(TM_BAD_INPUT, "null argument");
    submodel_sizes(*reinterpret_cast<SubModel*>(sm), out);
  });
}

tm_status tm_submodel_step(tm_sub* sm, double T, double dt, int32_t* converged, int32_t* newton, double* dMax) {
  return guarded([&] {
    if (!sm) fail(TM_BAD_INPUT, "null argument");
    int nw = 0;
    double dm = 0;
    const bool ok = submodel_step(*reinterpret_cast<SubModel*>(sm), T, dt, &nw, &dm);
    if (converged) *converged = ok;
    if (newton) *newton = nw;
    if (dMax) *dMax = dm;
  });
}

tm_status tm_submodel_get(tm_sub* sm, double* u, double* W, double* ebar) {
  return guarded([&] {
    if (!sm) fail(TM_BAD_INPUT, "null argument");
    submodel_get(*reinterpret_cast<SubModel*>(sm), u, W, ebar);
  });
}

// independent submodels (the sites of one die) over one history: the batched engine advances them
// together, every phase one launch over all of them
tm_status tm_submodel_run_batch(int32_t n, tm_sub* const* subs, int32_t nsteps, const double* t, const double* T, const int32_t* cycle,
                                int32_t cycles, const double* cphi, const double* sphi, double* out10, double* perCycle, double* loop,
                                int32_t* status) {
  return guarded([&] {
    if (n < 0 || (n > 0 && (!subs || !t || !T || !cycle || !cphi || !sphi || !out10 || !perCycle || !loop || !status)))
      fail(TM_BAD_INPUT, "null argument");
    std::vector<SubModel*> v(n);
    for (int i = 0; i < n; i++) {
      if (!subs[i]) fail(TM_BAD_INPUT, "null submodel");
      for (int j = 0; j < i; j++)
        if (subs[j] == subs[i]) fail(TM_BAD_INPUT, "a submodel appears twice in the batch");
      v[i] = reinterpret_cast<SubModel*>(subs[i]);
    }
    submodel_run_batch(v, nsteps, t, T, cycle, cycles, cphi, sphi, out10, perCycle, loop, status);
    for (int i = 0; i < n; i++)
      if (status[i] != TM_OK) fail((tm_status)status[i], "submodel " + std::to_string(i) + " of the batch failed");
  });
}

tm_status tm_submodel_run(tm_sub* sm, int32_t nsteps, const double* t, const double* T, const int32_t* cycle, int32_t cycles,
                          double cphi, double sphi, double* out10, double* perCycle, double* loop) {
  return guarded([&] {
    if (!sm || !t || !T || !cycle || !out10 || !perCycle || !loop) fail(TM_BAD_INPUT, "null argument");
    submodel_run(*reinterpret_cast<SubModel*>(sm), nsteps, t, T, cycle, cycles, cphi, sphi, out10, perCycle, loop);
  });
}

tm_status tm_submodel_run_sections(tm_sub* sm, int32_t nsteps, const double* t, const double* T, const int32_t* cycle,
                                   const int32_t* phase, int32_t cycles, double cphi, double sphi, double* out10, double* perCycle,
                                   double* loop, int32_t maxSnaps, int32_t* nSnaps, double* snapMeta, float* snapSig) {
  return guarded([&] {
    if (!sm || !t || !T || !cycle || !phase || !out10 || !perCycle || !loop || !nSnaps) fail(TM_BAD_INPUT, "null argument");
    submodel_run(*reinterpret_cast<SubModel*>(sm), nsteps, t, T, cycle, cycles, cphi, sphi, out10, perCycle, loop, phase, maxSnaps, nSnaps,
                 snapMeta, snapSig);
  });
}

tm_status tm_submodel_stress_snapshot(tm_sub* sm, double T, float* out) {
  return guarded([&] {
    if (!sm || !out) fail(TM_BAD_INPUT, "null argument");
    submodel_stress_snapshot(*reinterpret_cast<SubModel*>(sm), T, out);
  });
}

}  // extern "C"
