// Anand viscoplastic material point on the device (FP64), shared by the joint screening
// (tm_anand.cu) and the bump submodel (tm_submodel.cu). Include from files compiled without
// fused multiply-add: the operations then match the reference's JavaScript arithmetic.
//
// Follows src/core/13-fatigue.js:
//   AnandPoint._solveS   :32-52    inner scalar Newton on s with bisection safeguard
//   stepConstants        :61-65
//   AnandPoint.step      :67-143   backward-Euler J2 radial return, consistent tangent
//   _dsdd                :209-218
//   commit               :229-232
//
// The point functions are templates on the scalar type S: double for the screening and the
// submodel, Dual (tm_dual.cuh) for the forward-mode derivatives of a site's screening. The
// double instantiation is the same arithmetic as a plain double implementation.
#pragma once
#include <cmath>

#include "tm_dual.cuh"

namespace tmg {
namespace {

constexpr int ANAND_NEWTON_MAXIT = 60;
constexpr double ANAND_TOL = 1e-11;
constexpr int COLUMN_NEWTON_MAXIT = 20;
constexpr double COLUMN_STRESS_TOL = 1e-3;
constexpr double KELVIN = 273.15;
constexpr int TGRID_MIN = -80;
constexpr int TGRID_N = 381;

struct AnandConst {
  double A, QR, xi, m, shat, n, h0, a, s0, nu;
};

struct StepK {
  double G, K, expQ, rate0, dt;
};

__device__ __forceinline__ double sgn(double v) { return v > 0 ? 1.0 : (v < 0 ? -1.0 : 0.0); }

template <class S>
struct PointT {
  S ep[6], s, ebar, W, sigEq, lastD;
  S tr_ep[6], tr_s, tr_ebar, tr_W, tr_sigEq;
};
typedef PointT<double> Point;

template <class S>
__device__ S solve_s(const AnandConst& P, S s_n, S d, double dt, double expQ) {
  if (d <= 0) return s_n;
  const S sstar = P.shat * pow(d / (dt * P.A) * expQ, P.n);
  const S sn = s_n;
  const double h0 = P.h0, a = P.a;
  S lo = fmin(sn, sstar), hi = fmax(sn, sstar);
  if (hi - lo < 1e-14) return sn;
  S s = 0.5 * (lo + hi);
  for (int it = 0; it < ANAND_NEWTON_MAXIT; it++) {
    const S B0 = 1 - s / sstar;
    const S f = s - sn - h0 * pow(fabs(B0), a) * sgn(B0) * d;
    if (fabs(f) < ANAND_TOL * fmax(1.0, sn)) break;
    if (f > 0) hi = s; else lo = s;
    const S B = 1 - s / sstar;
    const S dphi = 1 + h0 * a * pow(fabs(B), a - 1) * d / sstar;
    S sn1 = s - f / dphi;
    if (!(sn1 > lo && sn1 < hi)) sn1 = 0.5 * (lo + hi);
    if (fabs(sn1 - s) < 1e-15 * fmax(1.0, s)) { s = sn1; break; }
    s = sn1;
  }
  return s;
}

template <class S>
__device__ S dsdd(const AnandConst& P, S d, S s, double dt, double expQ) {
  if (d <= 0) return S(0);
  const S sstar = P.shat * pow(d / (dt * P.A) * expQ, P.n);
  const S B = 1 - s / sstar;
  const S absB = fabs(B);
  const double sg = sgn(B);
  const double h0 = P.h0, a = P.a, n = P.n;
  const S dphi_ds = 1 + h0 * a * pow(absB, a - 1) * d / sstar;
  const S dphi_dd = -h0 * pow(absB, a) * sg - h0 * a * pow(absB, a - 1) * s * n / sstar;
  return -dphi_dd / dphi_ds;
}

__device__ double grid_at(const double* arr, double T) {
  const double x = T - TGRID_MIN;
  if (x <= 0) return arr[0];
  if (x >= TGRID_N - 1) return arr[TGRID_N - 1];
  const int i = (int)floor(x);
  const double t = x - i;
  const double a = arr[i], b = arr[i + 1];
  return a + t * (b - a);
}

__device__ StepK step_constants(const AnandConst& P, const double* Etab, double T, double dt) {
  const double E = grid_at(Etab, T), nu = P.nu;
  const double expQ = exp(P.QR / (T + KELVIN));
  StepK k;
  k.G = E / (2 * (1 + nu)); k.K = E / (3 * (1 - 2 * nu)); k.expQ = expQ; k.rate0 = dt * P.A / expQ; k.dt = dt;
  return k;
}

// AnandPoint.step (13-fatigue.js:67-143): fills sig (6) and D (36, when wantTangent)
template <class S>
__device__ S anand_step(const AnandConst& P, PointT<S>& pt, const S* eps, const StepK& k, S* sig, S* D, bool wantTangent) {
  const double G = k.G, K = k.K, expQ = k.expQ, rate0 = k.rate0, dt = k.dt;
  const S vol = (eps[0] + eps[1] + eps[2]) / 3;
  S e[6], str[6], nvec[6];
  e[0] = eps[0] - vol - pt.ep[0]; e[1] = eps[1] - vol - pt.ep[1]; e[2] = eps[2] - vol - pt.ep[2];
  e[3] = 0.5 * eps[3] - pt.ep[3]; e[4] = 0.5 * eps[4] - pt.ep[4]; e[5] = 0.5 * eps[5] - pt.ep[5];
  for (int i = 0; i < 6; i++) str[i] = 2 * G * e[i];
  const S nrm = sqrt(str[0] * str[0] + str[1] * str[1] + str[2] * str[2] + 2 * (str[3] * str[3] + str[4] * str[4] + str[5] * str[5]));
  const S sigTr = sqrt(1.5) * nrm;
  S d = 0, s1 = pt.s, dDdSig = 0;
  if (sigTr > 1e-14 && dt > 0) {
    const S dmax = sigTr / (3 * G);
    S lo = 0, hi = dmax;
    S dd = pt.lastD > 0 && pt.lastD < dmax ? pt.lastD : fmin(dmax, rate0 * pow(sinh(P.xi * sigTr / pt.s), 1 / P.m));
    if (!isfinite(dd) || dd <= 0) dd = 0.5 * dmax;
    S rg = 0, rs = pt.s, rx = 0, rsh = 0;
    for (int it = 0; it < ANAND_NEWTON_MAXIT; it++) {
      rs = solve_s(P, pt.s, dd, dt, expQ);
      rx = P.xi * (sigTr - 3 * G * dd) / rs;
      rsh = sinh(rx);
      rg = dd - rate0 * pow(rsh, 1 / P.m);
      if (!isfinite(rg)) { lo = dd; dd = 0.5 * (lo + hi); continue; }
      if (fabs(rg) < ANAND_TOL * fmax(dmax, 1e-30)) break;
      if (rg > 0) hi = dd; else lo = dd;
      const S fx = rate0 * (1 / P.m) * pow(rsh, 1 / P.m - 1) * cosh(rx);
      const S ds = dsdd(P, dd, rs, dt, expQ);
      const S sg = sigTr - 3 * G * dd;
      const S dg = 1 + fx * P.xi * (3 * G / rs + sg * ds / (rs * rs));
      S dn = dd - rg / dg;
      if (!(dn > lo && dn < hi) || !isfinite(dn)) dn = 0.5 * (lo + hi);
      if (fabs(dn - dd) < 1e-16 * fmax(dmax, 1e-30)) { dd = dn; break; }
      dd = dn;
    }
    d = dd; s1 = rs;
    pt.lastD = d;
    if (wantTangent) {
      const S fx = rate0 * (1 / P.m) * pow(rsh, 1 / P.m - 1) * cosh(rx);
      const S ds = dsdd(P, dd, rs, dt, expQ);
      const S sg = sigTr - 3 * G * dd;
      const S dg = 1 + fx * P.xi * (3 * G / rs + sg * ds / (rs * rs));
      dDdSig = (fx * P.xi / rs) / dg;
    }
  }
  const S theta = sigTr > 1e-14 ? 1 - 3 * G * d / sigTr : S(1);
  if (nrm > 0) for (int i = 0; i < 6; i++) nvec[i] = str[i] / nrm;
  else for (int i = 0; i < 6; i++) nvec[i] = 0;
  const S dg = sqrt(1.5) * d;
  for (int i = 0; i < 6; i++) pt.tr_ep[i] = pt.ep[i] + dg * nvec[i];
  const S sm = 3 * K * vol;
  sig[0] = theta * str[0] + sm; sig[1] = theta * str[1] + sm; sig[2] = theta * str[2] + sm;
  sig[3] = theta * str[3]; sig[4] = theta * str[4]; sig[5] = theta * str[5];
  const S sEq = sigTr - 3 * G * d;
  pt.tr_s = s1; pt.tr_ebar = pt.ebar + d; pt.tr_W = pt.W + 0.5 * (pt.sigEq + sEq) * d; pt.tr_sigEq = sEq;
  if (wantTangent) {
    const S thetaBar = 2 * G * 1.5 * dDdSig - (1 - theta);
    const S c1 = 2 * G * theta, c2 = 2 * G * thetaBar;
    for (int i = 0; i < 6; i++)
      for (int j = 0; j < 6; j++) {
        S v = -c2 * nvec[i] * nvec[j];
        if (i < 3 && j < 3) v += K + c1 * ((i == j ? 1 : 0) - 1.0 / 3);
        else if (i == j) v += 0.5 * c1;
        D[i * 6 + j] = v;
      }
  }
  return d;
}

template <class S>
__device__ void commit(PointT<S>& pt) {
  for (int i = 0; i < 6; i++) pt.ep[i] = pt.tr_ep[i];
  pt.s = pt.tr_s; pt.ebar = pt.tr_ebar; pt.W = pt.tr_W; pt.sigEq = pt.tr_sigEq;
}

}  // namespace
}  // namespace tmg
