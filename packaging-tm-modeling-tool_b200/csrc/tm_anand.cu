// Anand viscoplastic return map on the GPU (FP64): one thread per bump site integrates the
// whole cycle history, with the material state in registers.
//
// Follows src/core/13-fatigue.js:
//   AnandPoint._solveS   :32-52    inner scalar Newton on s with bisection safeguard
//   stepConstants        :61-65
//   AnandPoint.step      :67-143   backward-Euler J2 radial return, consistent tangent
//   stepColumn           :153-166  in-plane stresses of a free-standing column held at zero
//   stepSeriesColumn     :178-206  solder cap in series with an elastic pillar (screenDdi, :369-376)
//   _dsdd                :209-218
//   screenJoints loop    :395-451  strain interpolation, in-plane guesses, per-cycle W and ebar
// Compiled without fused multiply-add, like the reference's JavaScript arithmetic.
#include <atomic>
#include <cmath>
#include <exception>
#include <vector>

#include "tm_internal.h"
#include "tm_anand_point.cuh"

namespace tmg {

namespace {

template <class S>
__device__ void inv3(const S* J, S* out) {
  const S a = J[0], b = J[1], c = J[2], d = J[3], e = J[4], f = J[5], g = J[6], h = J[7], i = J[8];
  const S det = a * (e * i - f * h) - b * (d * i - f * g) + c * (d * h - e * g);
  out[0] = (e * i - f * h) / det; out[1] = (c * h - b * i) / det; out[2] = (b * f - c * e) / det;
  out[3] = (f * g - d * i) / det; out[4] = (a * i - c * g) / det; out[5] = (c * d - a * f) / det;
  out[6] = (d * h - e * g) / det; out[7] = (b * g - a * h) / det; out[8] = (a * e - b * d) / det;
}

// stepColumn (13-fatigue.js:153-166)
template <class S>
__device__ S step_column(const AnandConst& P, PointT<S>& pt, S* eps, const StepK& k, S* sig, S* D) {
  const int Pi[3] = {0, 1, 3};
  S A[9], Ai[9];
  S d = 0;
  for (int it = 0; it < COLUMN_NEWTON_MAXIT; it++) {
    d = anand_step(P, pt, (const S*)eps, k, sig, D, true);
    const S r0 = sig[0], r1 = sig[1], r2 = sig[3];
    const S ref = fmax(fmax(1.0, fabs(sig[2])), fmax(fabs(sig[4]), fabs(sig[5])));
    if (fmax(fmax(fabs(r0), fabs(r1)), fabs(r2)) < COLUMN_STRESS_TOL * ref) break;
    for (int r = 0; r < 3; r++)
      for (int c = 0; c < 3; c++) A[3 * r + c] = D[6 * Pi[r] + Pi[c]];
    inv3(A, Ai);
    for (int r = 0; r < 3; r++) eps[Pi[r]] -= Ai[3 * r] * r0 + Ai[3 * r + 1] * r1 + Ai[3 * r + 2] * r2;
  }
  return d;
}

// stepSeriesColumn (13-fatigue.js:178-206): the cap (height fraction fs) and a pillar of
// compliances Cp carry the same axial and shear stresses; tz = the prescribed column-average
// (zz, yz, zx) mechanical strains; the cap's in-plane stresses vanish. Newton on the cap's six
// strains, the 6x6 system by Gaussian elimination with partial pivoting.
template <class S>
__device__ S step_series_column(const AnandConst& P, PointT<S>& pt, S* eps, const S* tz, double fs, const double* Cp,
                                double E, const StepK& k, S* sig, S* D) {
  const int Pi[3] = {0, 1, 3}, Z[3] = {2, 4, 5}, ord[6] = {0, 1, 3, 2, 4, 5};
  const double fp = 1 - fs;
  S J[36], R[6];
  S d = 0;
  for (int it = 0; it < COLUMN_NEWTON_MAXIT; it++) {
    d = anand_step(P, pt, (const S*)eps, k, sig, D, true);
    for (int r = 0; r < 3; r++) {
      R[r] = sig[Pi[r]];
      R[3 + r] = fs * eps[Z[r]] + fp * Cp[r] * sig[Z[r]] - tz[r];
    }
    const S ref = fmax(fmax(1.0, fabs(sig[2])), fmax(fabs(sig[4]), fabs(sig[5])));
    S worst = 0;
    for (int r = 0; r < 3; r++) worst = fmax(fmax(worst, fabs(R[r])), fabs(R[3 + r]) * E);
    if (worst < COLUMN_STRESS_TOL * ref) break;
    for (int r = 0; r < 6; r++)
      for (int c = 0; c < 6; c++) {
        const S Dv = D[6 * ord[r] + ord[c]];
        J[6 * r + c] = r < 3 ? Dv : fp * Cp[r - 3] * Dv + (ord[r] == ord[c] ? fs : 0);
      }
    for (int c = 0; c < 6; c++) {
      int pr = c;
      for (int r = c + 1; r < 6; r++) if (fabs(J[6 * r + c]) > fabs(J[6 * pr + c])) pr = r;
      if (pr != c) {
        for (int q = 0; q < 6; q++) { const S t = J[6 * c + q]; J[6 * c + q] = J[6 * pr + q]; J[6 * pr + q] = t; }
        const S t = R[c]; R[c] = R[pr]; R[pr] = t;
      }
      const S piv = J[7 * c];
      for (int r = c + 1; r < 6; r++) {
        const S f = J[6 * r + c] / piv;
        if (f == 0) continue;
        for (int q = c; q < 6; q++) J[6 * r + q] -= f * J[6 * c + q];
        R[r] -= f * R[c];
      }
    }
    for (int c = 5; c >= 0; c--) {
      S v = R[c];
      for (int q = c + 1; q < 6; q++) v -= J[6 * c + q] * R[q];
      R[c] = v / J[7 * c];
    }
    for (int c = 0; c < 6; c++) eps[ord[c]] -= R[c];
  }
  return d;
}

// an elastic pillar under the solder cap: cap height fraction, per-step pillar compliances
// (1/E_p, 1/G_p, 1/G_p) and thermal strains, and the solder's E table (for the residual scale)
struct PillarArgs {
  double fs;
  const double* Cps;
  const double* Fp;
  const double* Etab;
};


// table entry i of a site: its value, and for the derivative kernel a unit derivative at the seeded entry
template <class S>
struct TabAt;
template <>
struct TabAt<double> {
  static __device__ __forceinline__ double at(const double* tab, int i, int) { return tab[i]; }
};
template <>
struct TabAt<Dual> {
  static __device__ __forceinline__ Dual at(const double* tab, int i, int seed) { return Dual(tab[i], i == seed ? 1.0 : 0.0); }
};

// screenJoints per-site loop (13-fatigue.js:416-451) for one site's strain table tab (ntemps x 6);
// SERIES: the joint is a solder cap on an elastic pillar (stepSeriesColumn), else a free-standing
// column (stepColumn). dW, dE: the last cycle's energy density and inelastic strain increments;
// stab: the cycle-to-cycle change of dW. For S = Dual the table entry `seed` carries a unit derivative.
template <class S, bool SERIES>
__device__ void screen_site(const AnandConst& P, const double* __restrict__ tab, int seed, int ntemps, int i25, int nsteps,
                            const int* __restrict__ wi, const double* __restrict__ wt, const double* __restrict__ Fth,
                            const StepK* __restrict__ kc, const double* __restrict__ Th, const int* __restrict__ cycle,
                            const int* __restrict__ phase, int cycles, const PillarArgs& pil, S& dWo, S& dEo, S& stabo) {
  typedef TabAt<S> TA;
  PointT<S> pt;
  for (int i = 0; i < 6; i++) pt.ep[i] = 0;
  pt.s = P.s0; pt.ebar = 0; pt.W = 0; pt.sigEq = 0; pt.lastD = 0;
  S e25[6], eps[6] = {0, 0, 0, 0, 0, 0}, e1[3] = {0, 0, 0}, e2[3] = {0, 0, 0}, sig[6], D[36];
  S s1[6] = {0, 0, 0, 0, 0, 0}, s2[6] = {0, 0, 0, 0, 0, 0};
  for (int c = 0; c < 6; c++) e25[c] = i25 >= 0 ? TA::at(tab, i25 * 6 + c, seed) : S(0);
  const int IP[3] = {0, 1, 3};
  const double nu = P.nu;
  // W and ebar at the end of the last three cycles (the reference keeps every cycle)
  S Wlast[3] = {0, 0, 0}, Elast[3] = {0, 0, 0};  // cycles nc-2, nc-1, nc
  for (int k = 1; k < nsteps; k++) {
    const int ia = wi[k] * 6, ib = ia + 6;
    const double t = wt[k];
    auto lerp = [&](int c) { const S av = TA::at(tab, ia + c, seed), bv = TA::at(tab, ib + c, seed); return av + t * (bv - av); };
    if (SERIES) {
      // column-average mechanical strain: the layer strain less the thermal strains of cap and pillar
      const double fs = pil.fs;
      S tz[3];
      tz[0] = lerp(2) - e25[2] - fs * Fth[k] - (1 - fs) * pil.Fp[k];
      tz[1] = lerp(4) - e25[4];
      tz[2] = lerp(5) - e25[5];
      if (k > 2 && phase[k] == phase[k - 1])
        for (int c = 0; c < 6; c++) eps[c] = 2 * s1[c] - s2[c];
      step_series_column(P, pt, eps, (const S*)tz, fs, pil.Cps + 3 * k, grid_at(pil.Etab, Th[k]), kc[k], sig, D);
      for (int c = 0; c < 6; c++) { s2[c] = s1[c]; s1[c] = eps[c]; }
    } else {
      const S ez = lerp(2) - e25[2] - Fth[k];
      if (k > 2 && phase[k] == phase[k - 1]) {
        for (int r = 0; r < 3; r++) eps[IP[r]] = 2 * e1[r] - e2[r];
      } else {
        eps[0] -= nu * (ez - eps[2]);
        eps[1] -= nu * (ez - eps[2]);
      }
      eps[2] = ez;
      eps[4] = lerp(4) - e25[4];
      eps[5] = lerp(5) - e25[5];
      step_column(P, pt, eps, kc[k], sig, D);
    }
    commit(pt);
    for (int r = 0; r < 3; r++) { e2[r] = e1[r]; e1[r] = eps[IP[r]]; }
    const int cyc = cycle[k];
    const int slot = cyc - (cycles - 2);
    if (slot >= 0 && slot < 3) { Wlast[slot] = pt.W; Elast[slot] = pt.ebar; }
  }
  // cycles before nc-2 stay 0 in the reference's per-cycle arrays when never reached
  const int nc = cycles;
  const S Wn = Wlast[2], Wn1 = nc - 1 >= 0 ? Wlast[1] : S(0), Wn2 = nc - 2 >= 0 ? Wlast[0] : S(0);
  dWo = Wn - Wn1;
  dEo = Elast[2] - Elast[1];
  stabo = nc >= 2 ? fabs((Wn - Wn1) - (Wn1 - Wn2)) / fmax(Wn - Wn1, 1e-30) : S(NAN);
}

// the screening, thread per site
template <bool SERIES>
__global__ void k_screen(AnandConst P, int nsites, int ntemps, int i25, const double* __restrict__ table, int nsteps,
                         const int* __restrict__ wi, const double* __restrict__ wt, const double* __restrict__ Fth,
                         const StepK* __restrict__ kc, const double* __restrict__ Th, const int* __restrict__ cycle,
                         const int* __restrict__ phase, int cycles, double* __restrict__ dW, double* __restrict__ dE,
                         double* __restrict__ stab, PillarArgs pil) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= nsites) return;
  const double* tab = table + (size_t)q * ntemps * 6;
  if (!isfinite(tab[0])) { dW[q] = NAN; dE[q] = NAN; stab[q] = NAN; return; }
  double w, e, st;
  screen_site<double, SERIES>(P, tab, -1, ntemps, i25, nsteps, wi, wt, Fth, kc, Th, cycle, phase, cycles, pil, w, e, st);
  dW[q] = w; dE[q] = e; stab[q] = st;
}

// derivatives of one site's last-cycle dW and dE with respect to every entry of its strain table:
// thread j runs the site's whole history with a unit derivative on table entry j (forward mode)
template <bool SERIES>
__global__ void k_screen_tangent(AnandConst P, int ntemps, int i25, const double* __restrict__ tab, int nsteps,
                                 const int* __restrict__ wi, const double* __restrict__ wt, const double* __restrict__ Fth,
                                 const StepK* __restrict__ kc, const double* __restrict__ Th, const int* __restrict__ cycle,
                                 const int* __restrict__ phase, int cycles, PillarArgs pil, double* __restrict__ out) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= 6 * ntemps) return;
  Dual w, e, st;
  screen_site<Dual, SERIES>(P, tab, j, ntemps, i25, nsteps, wi, wt, Fth, kc, Th, cycle, phase, cycles, pil, w, e, st);
  out[2 + j] = w.d;
  out[2 + 6 * ntemps + j] = e.d;
  if (j == 0) { out[0] = w.v; out[1] = e.v; }
}

__global__ void k_point_step(AnandConst P, const double* __restrict__ Etab, int npts, double* __restrict__ state,
                             const double* __restrict__ eps, double T, double dt, double* __restrict__ sig, double* __restrict__ D,
                             int commitFlag) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= npts) return;
  double* st = state + 12 * (size_t)q;
  Point pt;
  for (int i = 0; i < 6; i++) pt.ep[i] = st[i];
  pt.s = st[6]; pt.ebar = st[7]; pt.W = st[8]; pt.sigEq = st[9]; pt.lastD = st[10];
  const StepK k = step_constants(P, Etab, T, dt);
  double Dl[36];
  anand_step(P, pt, eps + 6 * (size_t)q, k, sig + 6 * (size_t)q, D ? D + 36 * (size_t)q : Dl, true);
  if (commitFlag) commit(pt);
  for (int i = 0; i < 6; i++) st[i] = pt.ep[i];
  st[6] = pt.s; st[7] = pt.ebar; st[8] = pt.W; st[9] = pt.sigEq; st[10] = pt.lastD;
}

__global__ void k_step_constants(AnandConst P, const double* __restrict__ Etab, int nsteps, const double* __restrict__ t,
                                 const double* __restrict__ T, StepK* __restrict__ kc) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nsteps) return;
  if (k == 0) { kc[0] = StepK{0, 0, 0, 0, 0}; return; }
  kc[k] = step_constants(P, Etab, T[k], t[k] - t[k - 1]);
}

AnandConst to_const(const tm_anand_material& m) {
  return AnandConst{m.A, m.QR, m.xi, m.m, m.shat, m.n, m.h0, m.a, m.s0, m.nu};
}

double grid_at_host(const double* arr, double T) {
  const double x = T - TGRID_MIN;
  if (x <= 0) return arr[0];
  if (x >= TGRID_N - 1) return arr[TGRID_N - 1];
  const int i = (int)std::floor(x);
  const double t = x - i;
  return arr[i] + t * (arr[i + 1] - arr[i]);
}

}  // namespace

void anand_screen_device(const tm_anand_material& mat, int nsites, int ntemps, const double* temps, const double* table_d, int nsteps,
                         const double* t_h, const double* T_h, const int* cycle_h, const int* phase_h, int cycles, double* dW_d,
                         double* dE_d, double* stab_d, cudaStream_t s, const tm_pillar* pillar, double* grad_d) {
  if (nsteps < 2 || ntemps < 2 || cycles < 1) fail(TM_BAD_INPUT, "anand screening: need >= 2 time steps, >= 2 temperatures, >= 1 cycle");
  if (pillar && (!(pillar->fs > 0 && pillar->fs <= 1) || !pillar->Etab || !pillar->Ftab))
    fail(TM_BAD_INPUT, "anand screening: the pillar needs a solder fraction in (0, 1] and its E and thermal strain tables");
  for (int k = 0; k < nsteps; k++)
    if (cycle_h[k] < 0 || cycle_h[k] > cycles) fail(TM_BAD_INPUT, "anand screening: cycle index out of range");
  int i25 = -1;
  for (int i = 0; i < ntemps; i++) if (temps[i] == 25) { i25 = i; break; }
  // per-step interpolation weights and thermal strains (13-fatigue.js:395-401)
  std::vector<int> wi(nsteps);
  std::vector<double> wt(nsteps), Fth(nsteps);
  for (int k = 0; k < nsteps; k++) {
    int i;
    if (T_h[k] <= temps[0]) i = 0;
    else if (T_h[k] >= temps[ntemps - 1]) i = ntemps - 2;
    else {
      int lo = 0, hi = ntemps - 1;
      while (hi - lo > 1) { const int mid = (lo + hi) >> 1; if (temps[mid] <= T_h[k]) lo = mid; else hi = mid; }
      i = lo;
    }
    wi[k] = i;
    const double tt = (T_h[k] - temps[i]) / (temps[i + 1] - temps[i]);
    wt[k] = tt < 0 ? 0 : (tt > 1 ? 1 : tt);
    Fth[k] = grid_at_host(mat.Ftab, T_h[k]) - grid_at_host(mat.Ftab, 25);
  }
  // a pillar in series: its compliances and thermal strain at every step (13-fatigue.js:410-414)
  std::vector<double> Cps, Fp;
  if (pillar) {
    Cps.resize(3 * (size_t)nsteps); Fp.resize(nsteps);
    for (int k = 0; k < nsteps; k++) {
      const double Ep = grid_at_host(pillar->Etab, T_h[k]), Gp = Ep / (2 * (1 + pillar->nu));
      if (!(Ep > 0) || !std::isfinite(Gp)) fail(TM_BAD_INPUT, "anand screening: pillar modulus must be positive");
      Cps[3 * k] = 1 / Ep; Cps[3 * k + 1] = Cps[3 * k + 2] = 1 / Gp;
      Fp[k] = grid_at_host(pillar->Ftab, T_h[k]) - grid_at_host(pillar->Ftab, 25);
    }
  }
  DBuf<int> d_wi, d_cycle, d_phase;
  DBuf<double> d_wt, d_Fth, d_t, d_T, d_E, d_Cps, d_Fp;
  DBuf<StepK> d_kc;
  d_wi.upload(wi, s); d_wt.upload(wt, s); d_Fth.upload(Fth, s);
  d_cycle.upload(cycle_h, nsteps, s); d_phase.upload(phase_h, nsteps, s);
  d_t.upload(t_h, nsteps, s); d_T.upload(T_h, nsteps, s); d_E.upload(mat.Etab, TGRID_N, s);
  d_kc.alloc(nsteps);
  const AnandConst P = to_const(mat);
  k_step_constants<<<(nsteps + 127) / 128, 128, 0, s>>>(P, d_E.p, nsteps, d_t.p, d_T.p, d_kc.p);
  if (grad_d) {
    // one site's dW and dE and their derivatives with respect to its table: thread per table entry
    PillarArgs pa{1, nullptr, nullptr, nullptr};
    if (pillar) { d_Cps.upload(Cps, s); d_Fp.upload(Fp, s); pa = PillarArgs{pillar->fs, d_Cps.p, d_Fp.p, d_E.p}; }
    const int nj = 6 * ntemps;
    if (pillar)
      k_screen_tangent<true><<<(nj + 63) / 64, 64, 0, s>>>(P, ntemps, i25, table_d, nsteps, d_wi.p, d_wt.p, d_Fth.p, d_kc.p, d_T.p,
                                                         d_cycle.p, d_phase.p, cycles, pa, grad_d);
    else
      k_screen_tangent<false><<<(nj + 63) / 64, 64, 0, s>>>(P, ntemps, i25, table_d, nsteps, d_wi.p, d_wt.p, d_Fth.p, d_kc.p, d_T.p,
                                                          d_cycle.p, d_phase.p, cycles, pa, grad_d);
  } else if (pillar) {
    d_Cps.upload(Cps, s); d_Fp.upload(Fp, s);
    const PillarArgs pa{pillar->fs, d_Cps.p, d_Fp.p, d_E.p};
    k_screen<true><<<(nsites + 63) / 64, 64, 0, s>>>(P, nsites, ntemps, i25, table_d, nsteps, d_wi.p, d_wt.p, d_Fth.p, d_kc.p, d_T.p,
                                                    d_cycle.p, d_phase.p, cycles, dW_d, dE_d, stab_d, pa);
  } else {
    k_screen<false><<<(nsites + 63) / 64, 64, 0, s>>>(P, nsites, ntemps, i25, table_d, nsteps, d_wi.p, d_wt.p, d_Fth.p, d_kc.p, d_T.p,
                                                     d_cycle.p, d_phase.p, cycles, dW_d, dE_d, stab_d, PillarArgs{1, nullptr, nullptr, nullptr});
  }
  note_launch(2);
  TM_CUDA_CHECK(cudaGetLastError());
  TM_CUDA_CHECK(cudaStreamSynchronize(s));
}

void anand_step_device(const tm_anand_material& mat, int npts, double* state_d, const double* eps_d, double T, double dt, double* sig_d,
                       double* D_d, int commitFlag, cudaStream_t s) {
  DBuf<double> d_E;
  d_E.upload(mat.Etab, TGRID_N, s);
  note_launch();
  k_point_step<<<(npts + 127) / 128, 128, 0, s>>>(to_const(mat), d_E.p, npts, state_d, eps_d, T, dt, sig_d, D_d, commitFlag);
  TM_CUDA_CHECK(cudaGetLastError());
  TM_CUDA_CHECK(cudaStreamSynchronize(s));
}

}  // namespace tmg

// ---- screening without device allocation -----------------------------------------------------------
// Some callers cannot allocate device memory at the time they screen: a host application whose
// allocator already owns the device memory (a caching allocator, or a process held to a fixed
// memory budget), or one that forbids allocations after start-up because cudaMalloc/cudaFree
// synchronize the device. For them, tm_anand_screen_noalloc keeps its per-step tables in this
// fixed array, which every GPU that loads the library holds until the process exits.
namespace tmg {
namespace {

constexpr int NA_STEPS = TM_NOALLOC_MAX_STEPS;
constexpr int NA_TEMPS = TM_NOALLOC_MAX_TEMPS;
// byte offsets of the tables inside the array (every table 256-byte aligned)
constexpr size_t NA_ALIGN(size_t b) { return (b + 255) / 256 * 256; }
constexpr size_t NA_KC = 0;
constexpr size_t NA_WT = NA_KC + NA_ALIGN(sizeof(StepK) * NA_STEPS);
constexpr size_t NA_FTH = NA_WT + NA_ALIGN(sizeof(double) * NA_STEPS);
constexpr size_t NA_TT = NA_FTH + NA_ALIGN(sizeof(double) * NA_STEPS);
constexpr size_t NA_TK = NA_TT + NA_ALIGN(sizeof(double) * NA_STEPS);
constexpr size_t NA_WI = NA_TK + NA_ALIGN(sizeof(double) * NA_STEPS);
constexpr size_t NA_CYC = NA_WI + NA_ALIGN(sizeof(int) * NA_STEPS);
constexpr size_t NA_PH = NA_CYC + NA_ALIGN(sizeof(int) * NA_STEPS);
constexpr size_t NA_TEMPSOFF = NA_PH + NA_ALIGN(sizeof(int) * NA_STEPS);
constexpr size_t NA_ETAB = NA_TEMPSOFF + NA_ALIGN(sizeof(double) * NA_TEMPS);
constexpr size_t NA_FTAB = NA_ETAB + NA_ALIGN(sizeof(double) * TGRID_N);
constexpr size_t NA_BYTES = NA_FTAB + NA_ALIGN(sizeof(double) * TGRID_N);

static __device__ __align__(256) unsigned char g_noalloc_scratch[NA_BYTES];

// device address of g_noalloc_scratch per device, looked up once per device with it current;
// atomic, since two host threads may make their first call on a device at the same moment (both
// store the same address)
constexpr int NA_MAX_DEVICES = 64;
std::atomic<unsigned char*> g_noalloc_addr[NA_MAX_DEVICES];

unsigned char* noalloc_scratch_address() {
  int dev = 0;
  TM_CUDA_CHECK(cudaGetDevice(&dev));
  if (dev < 0 || dev >= NA_MAX_DEVICES) fail(TM_BAD_INPUT, "device index beyond the no-allocation scratch table");
  unsigned char* a = g_noalloc_addr[dev].load(std::memory_order_acquire);
  if (!a) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) fail(TM_CUDA, std::string("cudaGetSymbolAddress of the screening scratch: ") + cudaGetErrorString(e));
    a = static_cast<unsigned char*>(p);
    g_noalloc_addr[dev].store(a, std::memory_order_release);
  }
  return a;
}

// per-step interpolation weights and thermal strains of screenJoints (13-fatigue.js:395-401), on the device
__global__ void k_step_weights(int nsteps, int ntemps, const double* __restrict__ temps, const double* __restrict__ T,
                               const double* __restrict__ Ftab, int* __restrict__ wi, double* __restrict__ wt, double* __restrict__ Fth) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nsteps) return;
  const double Tk = T[k];
  int i;
  if (Tk <= temps[0]) i = 0;
  else if (Tk >= temps[ntemps - 1]) i = ntemps - 2;
  else {
    int lo = 0, hi = ntemps - 1;
    while (hi - lo > 1) { const int mid = (lo + hi) >> 1; if (temps[mid] <= Tk) lo = mid; else hi = mid; }
    i = lo;
  }
  wi[k] = i;
  const double tt = (Tk - temps[i]) / (temps[i + 1] - temps[i]);
  wt[k] = tt < 0 ? 0 : (tt > 1 ? 1 : tt);
  Fth[k] = grid_at(Ftab, Tk) - grid_at(Ftab, 25);
}

}  // namespace
}  // namespace tmg

extern "C" tm_status tm_anand_screen_noalloc(const tm_anand_material* mat, int32_t nsites, int32_t ntemps, const double* temps,
                                             const double* table_dev, int32_t nsteps, const double* t, const double* T,
                                             const int32_t* cycle, const int32_t* phase, int32_t cycles, double* dW_dev,
                                             double* dE_dev, double* stab_dev, void* stream) {
  using namespace tmg;
  try {
    if (!mat || !temps || !table_dev || !t || !T || !cycle || !phase || !dW_dev || !dE_dev || !stab_dev)
      fail(TM_BAD_INPUT, "null argument");
    if (nsteps < 2 || ntemps < 2 || cycles < 1) fail(TM_BAD_INPUT, "anand screening: need >= 2 time steps, >= 2 temperatures, >= 1 cycle");
    if (nsteps > NA_STEPS) fail(TM_BAD_INPUT, "tm_anand_screen_noalloc: more than TM_NOALLOC_MAX_STEPS time steps");
    if (ntemps > NA_TEMPS) fail(TM_BAD_INPUT, "tm_anand_screen_noalloc: more than TM_NOALLOC_MAX_TEMPS temperatures");
    for (int k = 0; k < nsteps; k++)
      if (cycle[k] < 0 || cycle[k] > cycles) fail(TM_BAD_INPUT, "anand screening: cycle index out of range");
    if (nsites <= 0) return TM_OK;
    int i25 = -1;
    for (int i = 0; i < ntemps; i++) if (temps[i] == 25) { i25 = i; break; }
    require_device();
    unsigned char* base = noalloc_scratch_address();
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    StepK* kc = reinterpret_cast<StepK*>(base + NA_KC);
    double* wt = reinterpret_cast<double*>(base + NA_WT);
    double* Fth = reinterpret_cast<double*>(base + NA_FTH);
    double* tt = reinterpret_cast<double*>(base + NA_TT);
    double* Tk = reinterpret_cast<double*>(base + NA_TK);
    int* wi = reinterpret_cast<int*>(base + NA_WI);
    int* cyc = reinterpret_cast<int*>(base + NA_CYC);
    int* ph = reinterpret_cast<int*>(base + NA_PH);
    double* tmp = reinterpret_cast<double*>(base + NA_TEMPSOFF);
    double* Et = reinterpret_cast<double*>(base + NA_ETAB);
    double* Ft = reinterpret_cast<double*>(base + NA_FTAB);
    TM_CUDA_CHECK(cudaMemcpyAsync(tt, t, sizeof(double) * nsteps, cudaMemcpyHostToDevice, s));
    TM_CUDA_CHECK(cudaMemcpyAsync(Tk, T, sizeof(double) * nsteps, cudaMemcpyHostToDevice, s));
    TM_CUDA_CHECK(cudaMemcpyAsync(cyc, cycle, sizeof(int) * nsteps, cudaMemcpyHostToDevice, s));
    TM_CUDA_CHECK(cudaMemcpyAsync(ph, phase, sizeof(int) * nsteps, cudaMemcpyHostToDevice, s));
    TM_CUDA_CHECK(cudaMemcpyAsync(tmp, temps, sizeof(double) * ntemps, cudaMemcpyHostToDevice, s));
    TM_CUDA_CHECK(cudaMemcpyAsync(Et, mat->Etab, sizeof(double) * TGRID_N, cudaMemcpyHostToDevice, s));
    TM_CUDA_CHECK(cudaMemcpyAsync(Ft, mat->Ftab, sizeof(double) * TGRID_N, cudaMemcpyHostToDevice, s));
    const AnandConst P = to_const(*mat);
    k_step_constants<<<(nsteps + 127) / 128, 128, 0, s>>>(P, Et, nsteps, tt, Tk, kc);
    k_step_weights<<<(nsteps + 127) / 128, 128, 0, s>>>(nsteps, ntemps, tmp, Tk, Ft, wi, wt, Fth);
    k_screen<false><<<(nsites + 63) / 64, 64, 0, s>>>(P, nsites, ntemps, i25, table_dev, nsteps, wi, wt, Fth, kc, Tk, cyc, ph, cycles,
                                                     dW_dev, dE_dev, stab_dev, PillarArgs{1, nullptr, nullptr, nullptr});
    note_launch(3);
    TM_CUDA_CHECK(cudaGetLastError());
    TM_CUDA_CHECK(cudaStreamSynchronize(s));
    return TM_OK;
  } catch (const Error& e) {
    set_last_error(e.msg);
    return e.status;
  } catch (const std::exception& e) {
    set_last_error(e.what());
    return TM_CUDA;
  }
}
