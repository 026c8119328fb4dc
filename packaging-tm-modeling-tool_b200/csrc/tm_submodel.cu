// Bump submodel on the GPU (FP64): one pitch cell around a bump meshed with B-bar hexes, its
// cut boundary moved with the global fields, Anand solder Gauss points and incremental elastic
// parts, Newton with the algorithmic tangent and IC(0)-PCG inner solves, adaptive sub-steps
// over the cycle history, the hysteresis sampler and the per-cycle inelastic work of the two
// interface layers.
//
// Follows src/core/13-fatigue.js (BumpSubmodel):
//   constructor, _blockMap, _bbarCache   :518-608   grid, block map, B-bar matrices per element size
//   _boundary / prescribe                :646-694   boundary nodes, trilinear interpolation of fieldAt
//   _elastic / _elasRec                  :702-773   step-mean D and thermal stress increment per material
//   assemble                             :776-853   tangent and internal force (k_sub_assemble + gathers)
//   _commitElastic                       :856-872
//   _constrain                           :874-883
//   _solve                               :886-917   Jacobi-scaled IC(0)-PCG (tm_ic0.cu)
//   stepTo                               :924-956
//   _snapshot / _restore                 :994-1002
//   run                                  :1004-1104  sub-steps, sampleLoop, per-cycle W and ebar
//
// Every element is one warp: the lanes share the element's 24 x 24 matrix in shared memory and
// every entry is summed in the reference's order, as are the assembled blocks (gathered per
// block in element order) and the internal forces (gathered per node in element order), so the
// tangent and the residual of one Newton iteration are the reference's for the same state. The
// inner PCG sums its dots in a fixed order of its own. Compiled without fused multiply-add.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include <math_constants.h>

#include "tm_internal.h"
#include "tm_anand_point.cuh"

namespace tmg {

namespace {

constexpr double SUB_T_AVG = 0.025;          // 00-constants.js:114
constexpr int SUB_NEWTON_MAXIT = 25;         // :116
constexpr double SUB_RES_TOL = 1e-6;         // :117
constexpr double SUB_DU_TOL = 1e-8;          // :118
constexpr double SUB_INNER_TOL = 1e-8;       // :119
constexpr double INELASTIC_STEP_MAX = 2e-4;  // :113
constexpr int SA_WARPS = 4;                  // elements (warps) per block of the element kernels
enum { M_SUB = 0, M_SOLDER = 1, M_UF = 2, M_SI = 3 };

inline int blocks_for(size_t n, int per) { return (int)((n + per - 1) / per); }

// ---- host helpers: the material integrals of a step (03-materials.js:347-418) ------------------
double grid_at_s(const double* arr, double T, int stride, int comp) {
  const double x = T - TGRID_MIN;
  if (x <= 0) return arr[comp];
  if (x >= TGRID_N - 1) return arr[(TGRID_N - 1) * stride + comp];
  const int i = (int)std::floor(x);
  const double t = x - i;
  const double a = arr[i * stride + comp], b = arr[(i + 1) * stride + comp];
  return a + t * (b - a);
}
void grid_add_at(const double* grid, double T, int stride, int n, double w, double* out) {
  double x = T - TGRID_MIN;
  x = x < 0 ? 0 : (x > TGRID_N - 1 ? TGRID_N - 1 : x);
  const int i = std::min((int)std::floor(x), TGRID_N - 2);
  const double t = x - i;
  const int a = i * stride, b = a + stride;
  for (int c = 0; c < n; c++) out[c] += w * (grid[a + c] + t * (grid[b + c] - grid[a + c]));
}
template <class F> void for_grid_segments(double Ta, double Tb, F fn) {
  const double lo = std::min(Ta, Tb), hi = std::max(Ta, Tb);
  for (double t0 = lo; t0 < hi - 1e-12;) {
    const double t1 = std::min(hi, TGRID_MIN + std::floor(t0 - TGRID_MIN + 1e-9) + 1);
    fn(0.5 * (t0 + t1), t0, t1);
    t0 = t1;
  }
}
void grid_mean(const double* grid, int stride, int n, double Ta, double Tb, double* out) {
  for (int c = 0; c < n; c++) out[c] = 0;
  const double L = std::fabs(Tb - Ta);
  if (L < 1e-12) { grid_add_at(grid, Ta, stride, n, 1, out); return; }
  for_grid_segments(Ta, Tb, [&](double tm, double t0, double t1) { grid_add_at(grid, tm, stride, n, (t1 - t0) / L, out); });
}
void grid_stress_increment(const double* Dg, const double* Fg, double Ta, double Tb, double* out) {
  for (int r = 0; r < 6; r++) out[r] = 0;
  const double sg = Tb >= Ta ? 1 : -1;
  double D[36];
  for_grid_segments(Ta, Tb, [&](double tm, double t0, double t1) {
    for (auto& v : D) v = 0;
    grid_add_at(Dg, tm, 36, 36, 1, D);
    const double f0 = grid_at_s(Fg, t1, 3, 0) - grid_at_s(Fg, t0, 3, 0), f1 = grid_at_s(Fg, t1, 3, 1) - grid_at_s(Fg, t0, 3, 1),
                 f2 = grid_at_s(Fg, t1, 3, 2) - grid_at_s(Fg, t0, 3, 2);
    for (int r = 0; r < 6; r++) out[r] += sg * (D[6 * r] * f0 + D[6 * r + 1] * f1 + D[6 * r + 2] * f2);
  });
}
double grid_modulus_strain_increment(const double* E, const double* F, double Ta, double Tb) {
  const double sg = Tb >= Ta ? 1 : -1;
  double s = 0;
  for_grid_segments(Ta, Tb, [&](double tm, double t0, double t1) {
    s += grid_at_s(E, tm, 1, 0) * (grid_at_s(F, t1, 1, 0) - grid_at_s(F, t0, 1, 0));
  });
  return sg * s;
}
// columnD (03-materials.js:259-266): the solder phase of the bump layer as separate columns,
// in-plane terms at COLUMN_INPLANE_FRACTION (00-constants.js:25) of the axial ones
void column_d(double E, double nu, double* out) {
  const double fl = 1e-3, G = E / (2 * (1 + nu));
  for (int q = 0; q < 36; q++) out[q] = 0;
  out[0] = out[7] = fl * E;
  out[21] = fl * G;
  out[14] = E; out[28] = G; out[35] = G;
}

// isoD through isoEC and orthoD (03-materials.js:222-249), invDense (01-util.js:110-134)
void iso_d(double E, double nu, double nuMax, double* out) {
  const double nc = std::min(nu, nuMax);
  const double G = E / (2 * (1 + nc));
  const double S[9] = {1 / E, -nc / E, -nc / E, -nc / E, 1 / E, -nc / E, -nc / E, -nc / E, 1 / E};
  double M[18];
  for (int i = 0; i < 3; i++) for (int j = 0; j < 6; j++) M[i * 6 + j] = j < 3 ? S[i * 3 + j] : (j - 3 == i ? 1 : 0);
  for (int c = 0; c < 3; c++) {
    int p = c;
    double best = std::fabs(M[c * 6 + c]);
    for (int r = c + 1; r < 3; r++) { const double v = std::fabs(M[r * 6 + c]); if (v > best) { best = v; p = r; } }
    if (best == 0) fail(TM_BAD_INPUT, "submodel: singular isotropic compliance");
    if (p != c) for (int j = 0; j < 6; j++) std::swap(M[c * 6 + j], M[p * 6 + j]);
    const double inv = 1 / M[c * 6 + c];
    for (int j = 0; j < 6; j++) M[c * 6 + j] *= inv;
    for (int r = 0; r < 3; r++) {
      if (r == c) continue;
      const double f = M[r * 6 + c];
      if (f == 0) continue;
      for (int j = 0; j < 6; j++) M[r * 6 + j] -= f * M[c * 6 + j];
    }
  }
  for (int q = 0; q < 36; q++) out[q] = 0;
  for (int i = 0; i < 3; i++) for (int j = 0; j < 3; j++) out[i * 6 + j] = M[i * 6 + 3 + j];
  out[21] = G; out[28] = G; out[35] = G;
}

// boxDerivs (07-element.js:19-30) and bbarMatrix (13-fatigue.js:474-491)
const int HX[8] = {-1, 1, 1, -1, -1, 1, 1, -1}, HY[8] = {-1, -1, 1, 1, -1, -1, 1, 1}, HZ[8] = {-1, -1, -1, -1, 1, 1, 1, 1};
void box_derivs(double hx, double hy, double hz, double xi, double eta, double zeta, double* dx, double* dy, double* dz) {
  const double sx = 2 / hx, sy = 2 / hy, sz = 2 / hz;
  for (int a = 0; a < 8; a++) {
    const double xa = HX[a], ya = HY[a], za = HZ[a];
    dx[a] = xa * (1 + ya * eta) * (1 + za * zeta) * 0.125 * sx;
    dy[a] = ya * (1 + xa * xi) * (1 + za * zeta) * 0.125 * sy;
    dz[a] = za * (1 + xa * xi) * (1 + ya * eta) * 0.125 * sz;
  }
}
void bbar_matrix(double hx, double hy, double hz, double xi, double eta, double zeta, double* Bb) {
  double dx[8], dy[8], dz[8], cx[8], cy[8], cz[8];
  box_derivs(hx, hy, hz, xi, eta, zeta, dx, dy, dz);
  box_derivs(hx, hy, hz, 0, 0, 0, cx, cy, cz);
  for (int q = 0; q < 144; q++) Bb[q] = 0;
  for (int a = 0; a < 8; a++) {
    const int c = 3 * a;
    const double ddx = (cx[a] - dx[a]) / 3, ddy = (cy[a] - dy[a]) / 3, ddz = (cz[a] - dz[a]) / 3;
    Bb[0 * 24 + c] = dx[a] + ddx; Bb[0 * 24 + c + 1] = ddy; Bb[0 * 24 + c + 2] = ddz;
    Bb[1 * 24 + c] = ddx; Bb[1 * 24 + c + 1] = dy[a] + ddy; Bb[1 * 24 + c + 2] = ddz;
    Bb[2 * 24 + c] = ddx; Bb[2 * 24 + c + 1] = ddy; Bb[2 * 24 + c + 2] = dz[a] + ddz;
    Bb[3 * 24 + c] = dy[a]; Bb[3 * 24 + c + 1] = dx[a];
    Bb[4 * 24 + c + 1] = dz[a]; Bb[4 * 24 + c + 2] = dy[a];
    Bb[5 * 24 + c] = dz[a]; Bb[5 * 24 + c + 2] = dx[a];
  }
}

// ---- device kernels ------------------------------------------------------------------------------
constexpr unsigned FULLMASK = 0xffffffffu;

// prescribe: boundary node q, fieldAt blended between global temperatures i and i+1
__device__ __forceinline__ void sub_prescribe_node(int q, const int* __restrict__ bNodes, const int* __restrict__ bGlob,
                                                   const double* __restrict__ bW, const double* __restrict__ fa,
                                                   const double* __restrict__ fb, double t, const double* __restrict__ u25,
                                                   double* __restrict__ u) {
  double ux = 0, uy = 0, uz = 0;
  for (int c = 0; c < 8; c++) {
    const int gn = bGlob[8 * q + c];
    const double w = bW[8 * q + c];
    const double tx = fa[3 * gn] + t * (fb[3 * gn] - fa[3 * gn]), ty = fa[3 * gn + 1] + t * (fb[3 * gn + 1] - fa[3 * gn + 1]),
                 tz = fa[3 * gn + 2] + t * (fb[3 * gn + 2] - fa[3 * gn + 2]);
    ux += w * (tx - u25[3 * gn]); uy += w * (ty - u25[3 * gn + 1]); uz += w * (tz - u25[3 * gn + 2]);
  }
  const int n = bNodes[q];
  u[3 * n] = ux; u[3 * n + 1] = uy; u[3 * n + 2] = uz;
}
__global__ void k_sub_prescribe(int nb, const int* __restrict__ bNodes, const int* __restrict__ bGlob, const double* __restrict__ bW,
                                const double* __restrict__ fa, const double* __restrict__ fb, double t, const double* __restrict__ u25,
                                double* __restrict__ u) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q < nb) sub_prescribe_node(q, bNodes, bGlob, bW, fa, fb, t, u25, u);
}

// the per-warp shared work space of the element assembly
struct AsmSmem {
  double K[576], DB[144], Sig[48], D[288], Ue[24];
};

// assemble element e by one warp: elastic elements build K_e, f_th once per step (fresh) and give
// f_e = f_n + K_e (u_e - u_n,e) - f_th; solder elements step their 8 Anand points (one lane each)
// and sum f_e and, with wantK, K_e = sum_g w B^T D_g B
__device__ __forceinline__ void sub_assemble_element(int e, int lane, AsmSmem& sm, const int* __restrict__ conn,
                                                     const int* __restrict__ eMat, const int* __restrict__ eBb,
                                                     const double* __restrict__ Bm, const double* __restrict__ Bw,
                                                     const int* __restrict__ eAn, Point* __restrict__ pts, const double* __restrict__ u,
                                                     const double* __restrict__ uN, const double* __restrict__ eFn,
                                                     double* __restrict__ eK, double* __restrict__ eF, double* __restrict__ fe,
                                                     double* __restrict__ dmaxE, const double* __restrict__ elas, int fresh, int wantK,
                                                     const AnandConst& P, const StepK& kc, double fSolder) {
  double* K = sm.K;
  double* DB = sm.DB;
  double* ue = sm.Ue;
  const double* B = Bm + (size_t)eBb[e] * 8 * 144;
  const double wt = Bw[eBb[e]];
  const int an = eAn[e];
  if (lane < 24) ue[lane] = u[3 * (size_t)conn[8 * (size_t)e + lane / 3] + lane % 3];
  __syncwarp();
  if (an < 0) {
    double* Kc = eK + 576 * (size_t)e;
    double* fc = eF + 24 * (size_t)e;
    if (fresh) {
      const double* D = elas + 42 * eMat[e];
      const double* sth = D + 36;
      for (int o = lane; o < 576; o += 32) K[o] = 0;
      double fcl = 0;
      __syncwarp();
      for (int g = 0; g < 8; g++) {
        const double* Bb = B + 144 * g;
        if (lane < 24) {
          double sum = 0;
          for (int r = 0; r < 6; r++) sum += Bb[r * 24 + lane] * sth[r];
          fcl += wt * sum;
        }
        for (int o = lane; o < 144; o += 32) {
          const int r = o / 24, c = o % 24;
          double sum = 0;
          for (int t = 0; t < 6; t++) sum += D[r * 6 + t] * Bb[t * 24 + c];
          DB[o] = sum;
        }
        __syncwarp();
        for (int o = lane; o < 576; o += 32) {
          const int a = o / 24, b = o % 24;
          if (b < a) continue;
          double sum = 0;
          for (int r = 0; r < 6; r++) sum += Bb[r * 24 + a] * DB[r * 24 + b];
          K[o] += wt * sum;
        }
        __syncwarp();
      }
      for (int o = lane; o < 576; o += 32) {
        const int a = o / 24, b = o % 24;
        Kc[o] = b < a ? K[b * 24 + a] : K[o];
      }
      if (lane < 24) fc[lane] = fcl;
      __syncwarp();
    }
    if (lane < 24) ue[lane] -= uN[3 * (size_t)conn[8 * (size_t)e + lane / 3] + lane % 3];
    __syncwarp();
    if (lane < 24) {
      double sum = eFn[24 * (size_t)e + lane] - fc[lane];
      for (int b = 0; b < 24; b++) sum += Kc[lane * 24 + b] * ue[b];
      fe[24 * (size_t)e + lane] = sum;
    }
    if (lane == 0) dmaxE[e] = 0;
    return;
  }
  // solder: the 8 Gauss points, one lane each
  double d = 0;
  if (lane < 8) {
    const double* Bb = B + 144 * lane;
    double eps[6];
    for (int r = 0; r < 6; r++) {
      double s = 0;
      for (int c = 0; c < 24; c++) s += Bb[r * 24 + c] * ue[c];
      eps[r] = s;
    }
    eps[0] -= fSolder; eps[1] -= fSolder; eps[2] -= fSolder;
    d = anand_step(P, pts[8 * (size_t)an + lane], eps, kc, sm.Sig + 6 * lane, sm.D + 36 * lane, wantK != 0);
  }
  for (int off = 16; off > 0; off >>= 1) d = fmax(d, __shfl_xor_sync(FULLMASK, d, off));
  if (lane == 0) dmaxE[e] = d;
  __syncwarp();
  if (lane < 24) {
    double f = 0;
    for (int g = 0; g < 8; g++) {
      const double* Bb = B + 144 * g;
      const double* sig = sm.Sig + 6 * g;
      double s = 0;
      for (int r = 0; r < 6; r++) s += Bb[r * 24 + lane] * sig[r];
      f += wt * s;
    }
    fe[24 * (size_t)e + lane] = f;
  }
  if (!wantK) return;
  for (int o = lane; o < 576; o += 32) K[o] = 0;
  __syncwarp();
  for (int g = 0; g < 8; g++) {
    const double* Bb = B + 144 * g;
    const double* Dg = sm.D + 36 * g;
    for (int o = lane; o < 144; o += 32) {
      const int r = o / 24, c = o % 24;
      double s = 0;
      for (int t = 0; t < 6; t++) s += Dg[r * 6 + t] * Bb[t * 24 + c];
      DB[o] = s;
    }
    __syncwarp();
    for (int o = lane; o < 576; o += 32) {
      const int a = o / 24, b = o % 24;
      if (b < a) continue;
      double s = 0;
      for (int r = 0; r < 6; r++) s += Bb[r * 24 + a] * DB[r * 24 + b];
      K[o] += wt * s;
    }
    __syncwarp();
  }
  double* Ke = eK + 576 * (size_t)e;
  for (int o = lane; o < 576; o += 32) {
    const int a = o / 24, b = o % 24;
    Ke[o] = b < a ? K[b * 24 + a] : K[o];
  }
}
__global__ void __launch_bounds__(32 * SA_WARPS)
k_sub_assemble(int ne, const int* __restrict__ conn, const int* __restrict__ eMat, const int* __restrict__ eBb, const double* __restrict__ Bm,
               const double* __restrict__ Bw, const int* __restrict__ eAn, Point* __restrict__ pts, const double* __restrict__ u,
               const double* __restrict__ uN, const double* __restrict__ eFn, double* __restrict__ eK, double* __restrict__ eF,
               double* __restrict__ fe, double* __restrict__ dmaxE, const double* __restrict__ elas, int fresh, int wantK, AnandConst P,
               StepK kc, double fSolder) {
  __shared__ AsmSmem sm[SA_WARPS];
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int e = blockIdx.x * SA_WARPS + w;
  if (e >= ne) return;
  sub_assemble_element(e, lane, sm[w], conn, eMat, eBb, Bm, Bw, eAn, pts, u, uN, eFn, eK, eF, fe, dmaxE, elas, fresh, wantK, P, kc, fSolder);
}

// the tangent's blocks, thread per block: the element contributions in element order, then the
// constrained rows and columns zeroed off the diagonal (_constrain)
__device__ __forceinline__ void sub_gather_val_block(int k, const int* __restrict__ blkRow, const int* __restrict__ col,
                                                     const int* __restrict__ start, const int* __restrict__ list,
                                                     const double* __restrict__ eK, const uint8_t* __restrict__ isC,
                                                     double* __restrict__ val) {
  const int i = blkRow[k], j = col[k];
  double v[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  for (int l = start[k]; l < start[k + 1]; l++) {
    const int code = list[l], e = code >> 6, a = (code >> 3) & 7, b = code & 7;
    const double* Ke = eK + 576 * (size_t)e;
    for (int p = 0; p < 3; p++)
      for (int q = 0; q < 3; q++) v[3 * p + q] += Ke[(3 * a + p) * 24 + 3 * b + q];
  }
  for (int p = 0; p < 3; p++)
    for (int q = 0; q < 3; q++) {
      const int r = 3 * i + p, c = 3 * j + q;
      if ((isC[r] || isC[c]) && r != c) v[3 * p + q] = 0;
      val[9 * (size_t)k + 3 * p + q] = v[3 * p + q];
    }
}
__global__ void k_sub_gather_val(int nb, const int* __restrict__ blkRow, const int* __restrict__ col, const int* __restrict__ start,
                                 const int* __restrict__ list, const double* __restrict__ eK, const uint8_t* __restrict__ isC,
                                 double* __restrict__ val) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < nb) sub_gather_val_block(k, blkRow, col, start, list, eK, isC, val);
}

// internal force, thread per DOF: the element forces in element order
__device__ __forceinline__ void sub_gather_rint_dof(int q, const int* __restrict__ start, const int* __restrict__ list,
                                                    const double* __restrict__ fe, double* __restrict__ rint) {
  const int n = q / 3, p = q % 3;
  double s = 0;
  for (int l = start[n]; l < start[n + 1]; l++) {
    const int code = list[l], e = code >> 3, a = code & 7;
    s += fe[24 * (size_t)e + 3 * a + p];
  }
  rint[q] = s;
}
__global__ void k_sub_gather_rint(int ndof, const int* __restrict__ start, const int* __restrict__ list, const double* __restrict__ fe,
                                  double* __restrict__ rint) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q < ndof) sub_gather_rint_dof(q, start, list, fe, rint);
}

// deterministic sums over one block: out[0..m) = sums of m products (pairs of arrays, or with a mask)
// kind 0: a.a over the free DOFs, a.a over all (the Newton residual norms)
// kind 1: a.b
// kind 2: after u += du on the free DOFs: du.du over the free DOFs, u.u over all
// deterministic sums over n entries: the entries are cut into sums_parts(n) contiguous slices (a
// function of n only), a CTA sums one slice by a strided loop and a fixed tree, and the slices'
// partial sums are added in slice order; two results per call (out[0], out[1]):
// kind 0: a.a over the free DOFs, a.a over all (the Newton residual norms)
// kind 1: a.b
// kind 2: after u += du on the free DOFs: du.du over the free DOFs, u.u over all
constexpr int SUMS_THREADS = 256;
constexpr int SUMS_SLICE = 16384;        // entries per slice, before the cap on the slice count
constexpr int SUMS_MAXP = 64;            // slices at most
__host__ __device__ inline int sums_parts(int n) {
  const int p = (n + SUMS_SLICE - 1) / SUMS_SLICE;
  return p < 1 ? 1 : (p > SUMS_MAXP ? SUMS_MAXP : p);
}
// slice c of n entries into part[2c], part[2c + 1]
__device__ __forceinline__ void sub_sums_slice(int n, int c, int kind, const double* __restrict__ a, double* __restrict__ b,
                                               const uint8_t* __restrict__ isC, double* __restrict__ part, double* s0, double* s1) {
  const int parts = sums_parts(n), len = (n + parts - 1) / parts;
  const int q0 = c * len, q1 = min(n, q0 + len);
  double x0 = 0, x1 = 0;
  for (int q = q0 + threadIdx.x; q < q1; q += SUMS_THREADS) {
    if (kind == 0) {
      const double v = a[q];
      if (!isC[q]) x0 += v * v;
      x1 += v * v;
    } else if (kind == 1) {
      x0 += a[q] * b[q];
    } else {
      if (!isC[q]) { b[q] += a[q]; x0 += a[q] * a[q]; }
      x1 += b[q] * b[q];
    }
  }
  s0[threadIdx.x] = x0; s1[threadIdx.x] = x1;
  __syncthreads();
  for (int h = SUMS_THREADS / 2; h > 0; h >>= 1) {
    if ((int)threadIdx.x < h) { s0[threadIdx.x] += s0[threadIdx.x + h]; s1[threadIdx.x] += s1[threadIdx.x + h]; }
    __syncthreads();
  }
  if (threadIdx.x == 0) { part[2 * c] = s0[0]; part[2 * c + 1] = s1[0]; }
}
__device__ __forceinline__ void sub_sums_final(int n, const double* __restrict__ part, double* __restrict__ out) {
  double x0 = 0, x1 = 0;
  for (int c = 0; c < sums_parts(n); c++) { x0 += part[2 * c]; x1 += part[2 * c + 1]; }
  out[0] = x0; out[1] = x1;
}
__global__ void __launch_bounds__(SUMS_THREADS) k_sub_sums_slice(int n, int kind, const double* __restrict__ a, double* __restrict__ b,
                                                                 const uint8_t* __restrict__ isC, double* __restrict__ part) {
  __shared__ double s0[SUMS_THREADS], s1[SUMS_THREADS];
  sub_sums_slice(n, blockIdx.x, kind, a, b, isC, part, s0, s1);
}
__global__ void k_sub_sums_final(int n, const double* __restrict__ part, double* __restrict__ out) {
  if (threadIdx.x == 0 && blockIdx.x == 0) sub_sums_final(n, part, out);
}

// _solve's scaling: s from the tangent's diagonal, the scaled copy, b = rhs s with rhs = -rint
// on the free DOFs
__device__ __forceinline__ void sub_scale_s_node(int i, const int* __restrict__ diag, const double* __restrict__ val,
                                                 double* __restrict__ s) {
  const double* v = val + 9 * (size_t)diag[i];
  s[3 * i] = 1 / sqrt(fmax(v[0], 1e-300)); s[3 * i + 1] = 1 / sqrt(fmax(v[4], 1e-300)); s[3 * i + 2] = 1 / sqrt(fmax(v[8], 1e-300));
}
__global__ void k_sub_scale_s(int nn, const int* __restrict__ diag, const double* __restrict__ val, double* __restrict__ s) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < nn) sub_scale_s_node(i, diag, val, s);
}
__device__ __forceinline__ void sub_scale_vals_block(int k, const int* __restrict__ blkRow, const int* __restrict__ col,
                                                     const double* __restrict__ s, const double* __restrict__ val,
                                                     double* __restrict__ vals) {
  const int i = blkRow[k], j = col[k];
  for (int p = 0; p < 3; p++)
    for (int q = 0; q < 3; q++) vals[9 * (size_t)k + 3 * p + q] = val[9 * (size_t)k + 3 * p + q] * (s[3 * i + p] * s[3 * j + q]);
}
__global__ void k_sub_scale_vals(int nb, const int* __restrict__ blkRow, const int* __restrict__ col, const double* __restrict__ s,
                                 const double* __restrict__ val, double* __restrict__ vals) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < nb) sub_scale_vals_block(k, blkRow, col, s, val, vals);
}
__device__ __forceinline__ void sub_rhs_dof(int q, const double* __restrict__ rint, const uint8_t* __restrict__ isC,
                                            const double* __restrict__ s, double* __restrict__ b, double* __restrict__ r,
                                            double* __restrict__ x) {
  const double rhs = isC[q] ? 0 : -rint[q];
  const double v = rhs * s[q];
  b[q] = v; r[q] = v; x[q] = 0;
}
__global__ void k_sub_rhs(int n, const double* __restrict__ rint, const uint8_t* __restrict__ isC, const double* __restrict__ s,
                          double* __restrict__ b, double* __restrict__ r, double* __restrict__ x) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q < n) sub_rhs_dof(q, rint, isC, s, b, r, x);
}
// fullMatVec (09-assembly.js:151-165), node i
__device__ __forceinline__ void sub_spmv_node(int i, const int* __restrict__ rowPtr, const int* __restrict__ col,
                                              const double* __restrict__ val, const double* __restrict__ x, double* __restrict__ y) {
  double y0 = 0, y1 = 0, y2 = 0;
  for (int k = rowPtr[i]; k < rowPtr[i + 1]; k++) {
    const int j = col[k];
    const double* v = val + 9 * (size_t)k;
    const double x0 = x[3 * j], x1 = x[3 * j + 1], x2 = x[3 * j + 2];
    y0 += v[0] * x0 + v[1] * x1 + v[2] * x2;
    y1 += v[3] * x0 + v[4] * x1 + v[5] * x2;
    y2 += v[6] * x0 + v[7] * x1 + v[8] * x2;
  }
  y[3 * i] = y0; y[3 * i + 1] = y1; y[3 * i + 2] = y2;
}
__global__ void k_sub_spmv(int nn, const int* __restrict__ rowPtr, const int* __restrict__ col, const double* __restrict__ val,
                           const double* __restrict__ x, double* __restrict__ y) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < nn) sub_spmv_node(i, rowPtr, col, val, x, y);
}
// the PCG updates with their scalars read on the device: alpha = rz / (p.q), beta = rz2 / rz
__device__ __forceinline__ void sub_axpy2_dof(int i, double rz, double pq, const double* __restrict__ p, const double* __restrict__ q,
                                              double* __restrict__ x, double* __restrict__ r) {
  const double alpha = rz / pq;
  x[i] += alpha * p[i];
  r[i] += -alpha * q[i];
}
__global__ void k_sub_axpy2(int n, const double* __restrict__ rz, const double* __restrict__ pq, const double* __restrict__ p,
                            const double* __restrict__ q, double* __restrict__ x, double* __restrict__ r) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) sub_axpy2_dof(i, *rz, *pq, p, q, x, r);
}
__device__ __forceinline__ void sub_xpby_dof(int i, double rz2, double rz, const double* __restrict__ z, double* __restrict__ p) {
  const double beta = rz2 / rz;
  p[i] = z[i] + beta * p[i];
}
__global__ void k_sub_xpby(int n, const double* __restrict__ z, const double* __restrict__ rz2, const double* __restrict__ rz,
                           double* __restrict__ p) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) sub_xpby_dof(i, *rz2, *rz, z, p);
}
// ---- z-line block-Jacobi preconditioner of the scaled tangent --------------------------------------
// The cell's nodes (i ny + j) nz + k form columns of nz consecutive ids. Per column the 3x3-block
// tridiagonal part of the scaled tangent (diagonal blocks and the couplings to the node below) is
// factored as L L^T, L block lower bidiagonal, and applied by a forward and a backward block
// substitution; all columns are independent, so one thread takes one column and one launch applies
// the whole preconditioner (an SPD block-Jacobi splitting: a valid PCG preconditioner). Per node
// 15 values: 1/l00, 1/l11, l10, 1/l22, l20, l21 of the diagonal factor, then the 3x3 coupling
// L_{k,k-1} row-major. A pivot that is not positive (the scaled tangent's diagonal is 1) is taken
// as 1e-12, so the factor exists for any tangent.
constexpr int LF_VALS = 15;
constexpr double LF_PIVOT_MIN = 1e-12;

__device__ __forceinline__ void sub_line_factor_column(int c, int nz, const int* __restrict__ diag, const int* __restrict__ subBlk,
                                                       const double* __restrict__ vals, double* __restrict__ lf) {
  double L[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};   // previous node's diagonal factor (lower, row-major)
  for (int k = 0; k < nz; k++) {
    const int n = c * nz + k;
    const double* A = vals + 9 * (size_t)diag[n];
    double a00 = A[0], a10 = A[3], a11 = A[4], a20 = A[6], a21 = A[7], a22 = A[8];
    double X[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    if (k > 0) {
      // X = C L_prev^-T: each row x of X solves L_prev x^T = c^T for the row c of C = A_{k,k-1}
      const double* Cb = vals + 9 * (size_t)subBlk[n];
      for (int r = 0; r < 3; r++) {
        const double c0 = Cb[3 * r], c1 = Cb[3 * r + 1], c2 = Cb[3 * r + 2];
        const double x0 = c0 / L[0];
        const double x1 = (c1 - L[3] * x0) / L[4];
        const double x2 = (c2 - L[6] * x0 - L[7] * x1) / L[8];
        X[3 * r] = x0; X[3 * r + 1] = x1; X[3 * r + 2] = x2;
      }
      a00 -= X[0] * X[0] + X[1] * X[1] + X[2] * X[2];
      a10 -= X[3] * X[0] + X[4] * X[1] + X[5] * X[2];
      a11 -= X[3] * X[3] + X[4] * X[4] + X[5] * X[5];
      a20 -= X[6] * X[0] + X[7] * X[1] + X[8] * X[2];
      a21 -= X[6] * X[3] + X[7] * X[4] + X[8] * X[5];
      a22 -= X[6] * X[6] + X[7] * X[7] + X[8] * X[8];
    }
    const double l00 = sqrt(fmax(a00, LF_PIVOT_MIN));
    const double l10 = a10 / l00, l20 = a20 / l00;
    const double l11 = sqrt(fmax(a11 - l10 * l10, LF_PIVOT_MIN));
    const double l21 = (a21 - l20 * l10) / l11;
    const double l22 = sqrt(fmax(a22 - l20 * l20 - l21 * l21, LF_PIVOT_MIN));
    double* f = lf + LF_VALS * (size_t)n;
    f[0] = 1 / l00; f[1] = 1 / l11; f[2] = l10; f[3] = 1 / l22; f[4] = l20; f[5] = l21;
    for (int q = 0; q < 9; q++) f[6 + q] = X[q];
    L[0] = l00; L[3] = l10; L[4] = l11; L[6] = l20; L[7] = l21; L[8] = l22;
  }
}

// z = M^-1 r on one column: y = L^-1 r downwards, z = L^-T y upwards
__device__ __forceinline__ void sub_line_apply_column(int c, int nz, const double* __restrict__ lf, const double* __restrict__ r,
                                                      double* __restrict__ z) {
  double y0 = 0, y1 = 0, y2 = 0;
  for (int k = 0; k < nz; k++) {
    const size_t n = (size_t)c * nz + k;
    const double* f = lf + LF_VALS * n;
    double b0 = r[3 * n], b1 = r[3 * n + 1], b2 = r[3 * n + 2];
    if (k > 0) {
      b0 -= f[6] * y0 + f[7] * y1 + f[8] * y2;
      b1 -= f[9] * y0 + f[10] * y1 + f[11] * y2;
      b2 -= f[12] * y0 + f[13] * y1 + f[14] * y2;
    }
    y0 = b0 * f[0];
    y1 = (b1 - f[2] * y0) * f[1];
    y2 = (b2 - f[4] * y0 - f[5] * y1) * f[3];
    z[3 * n] = y0; z[3 * n + 1] = y1; z[3 * n + 2] = y2;
  }
  double t0 = 0, t1 = 0, t2 = 0;   // L_{k+1,k}^T z_{k+1}
  for (int k = nz - 1; k >= 0; k--) {
    const size_t n = (size_t)c * nz + k;
    const double* f = lf + LF_VALS * n;
    const double b0 = z[3 * n] - t0, b1 = z[3 * n + 1] - t1, b2 = z[3 * n + 2] - t2;
    const double z2 = b2 * f[3];
    const double z1 = (b1 - f[5] * z2) * f[1];
    const double z0 = (b0 - f[2] * z1 - f[4] * z2) * f[0];
    z[3 * n] = z0; z[3 * n + 1] = z1; z[3 * n + 2] = z2;
    t0 = f[6] * z0 + f[9] * z1 + f[12] * z2;
    t1 = f[7] * z0 + f[10] * z1 + f[13] * z2;
    t2 = f[8] * z0 + f[11] * z1 + f[14] * z2;
  }
}
__global__ void k_sub_line_factor(int ncol, int nz, const int* __restrict__ diag, const int* __restrict__ subBlk,
                                  const double* __restrict__ vals, double* __restrict__ lf) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c < ncol) sub_line_factor_column(c, nz, diag, subBlk, vals, lf);
}
__global__ void k_sub_line_apply(int ncol, int nz, const double* __restrict__ lf, const double* __restrict__ r, double* __restrict__ z) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c < ncol) sub_line_apply_column(c, nz, lf, r, z);
}

__global__ void k_sub_mul(int n, const double* __restrict__ s, double* __restrict__ x) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) x[i] *= s[i];
}

// _commitElastic, warp per elastic element: Gauss-point stresses and the element's internal force
struct CommitSmem {
  double Due[24], Sg[6], De[6];
};
__device__ __forceinline__ void sub_commit_elastic_element(int e, int lane, CommitSmem& sm, const int* __restrict__ conn,
                                                           const int* __restrict__ eMat, const int* __restrict__ eBb,
                                                           const double* __restrict__ Bm, const double* __restrict__ Bw,
                                                           const double* __restrict__ u, const double* __restrict__ uN,
                                                           const double* __restrict__ elas, double* __restrict__ sigE,
                                                           double* __restrict__ eFn) {
  const double* D = elas + 42 * eMat[e];
  const double* sth = D + 36;
  const double* B = Bm + (size_t)eBb[e] * 8 * 144;
  const double wt = Bw[eBb[e]];
  double* due = sm.Due;
  if (lane < 24) {
    const size_t n = 3 * (size_t)conn[8 * (size_t)e + lane / 3] + lane % 3;
    due[lane] = u[n] - uN[n];
  }
  __syncwarp();
  double fn = 0;
  for (int g = 0; g < 8; g++) {
    const double* Bb = B + 144 * g;
    double* so = sigE + 48 * (size_t)e + 6 * g;
    if (lane < 6) {
      double s2 = 0;
      for (int c = 0; c < 24; c++) s2 += Bb[lane * 24 + c] * due[c];
      sm.De[lane] = s2;
    }
    __syncwarp();
    if (lane < 6) {
      double s2 = -sth[lane];
      for (int c = 0; c < 6; c++) s2 += D[lane * 6 + c] * sm.De[c];
      so[lane] += s2;
      sm.Sg[lane] = so[lane];
    }
    __syncwarp();
    if (lane < 24) {
      double s2 = 0;
      for (int r = 0; r < 6; r++) s2 += Bb[r * 24 + lane] * sm.Sg[r];
      fn += wt * s2;
    }
    __syncwarp();
  }
  if (lane < 24) eFn[24 * (size_t)e + lane] = fn;
}
__global__ void __launch_bounds__(32 * SA_WARPS)
k_sub_commit_elastic(int ne, const int* __restrict__ conn, const int* __restrict__ eMat, const int* __restrict__ eBb,
                     const double* __restrict__ Bm, const double* __restrict__ Bw, const int* __restrict__ eAn, const double* __restrict__ u,
                     const double* __restrict__ uN, const double* __restrict__ elas, double* __restrict__ sigE, double* __restrict__ eFn) {
  __shared__ CommitSmem sm[SA_WARPS];
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int e = blockIdx.x * SA_WARPS + w;
  if (e >= ne || eAn[e] >= 0) return;
  sub_commit_elastic_element(e, lane, sm[w], conn, eMat, eBb, Bm, Bw, u, uN, elas, sigE, eFn);
}

__global__ void k_sub_commit_points(int np, Point* __restrict__ pts) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < np) commit(pts[i]);
}

// GP_TO_NODE (07-element.js:227-234): nodal value = sum_g N_g(sqrt3 x node natural coords) v_g
struct GpToNode {
  double M[64];
};

// _stressSnapshot (13-fatigue.js:965-989), thread per element: the 48 nodal stresses (float32)
// extrapolated from the Gauss points: the committed Gauss-point stresses of elastic elements, and
// at solder points the stress of the current displacement at the committed plastic strain
// (AnandPoint.stressAt, :221-227); f the solder's thermal strain from 25 degC, E its modulus at T
__global__ void __launch_bounds__(128) k_sub_stress_snapshot(int ne, const int* __restrict__ conn, const int* __restrict__ eAn,
                                                             const int* __restrict__ eBb, const double* __restrict__ Bm,
                                                             const Point* __restrict__ pts, const double* __restrict__ u,
                                                             const double* __restrict__ sigE, double E, double nu, double f,
                                                             const GpToNode G2N, float* __restrict__ out) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= ne) return;
  double gp[48];
  if (eAn[e] < 0) {
    for (int q = 0; q < 48; q++) gp[q] = sigE[48 * (size_t)e + q];
  } else {
    double ue[24];
    for (int a = 0; a < 8; a++) {
      const int n = conn[8 * (size_t)e + a];
      ue[3 * a] = u[3 * (size_t)n]; ue[3 * a + 1] = u[3 * (size_t)n + 1]; ue[3 * a + 2] = u[3 * (size_t)n + 2];
    }
    const double G = E / (2 * (1 + nu)), K = E / (3 * (1 - 2 * nu));
    const double* Ball = Bm + (size_t)eBb[e] * 8 * 144;
    for (int g = 0; g < 8; g++) {
      const double* Bb = Ball + 144 * g;
      double eps[6];
      for (int r = 0; r < 6; r++) {
        double sm = 0;
        for (int c = 0; c < 24; c++) sm += Bb[r * 24 + c] * ue[c];
        eps[r] = sm;
      }
      eps[0] -= f; eps[1] -= f; eps[2] -= f;
      const Point& pt = pts[8 * (size_t)eAn[e] + g];
      const double vol = (eps[0] + eps[1] + eps[2]) / 3, smv = 3 * K * vol;
      for (int i = 0; i < 3; i++) gp[6 * g + i] = 2 * G * (eps[i] - vol - pt.ep[i]) + smv;
      for (int i = 3; i < 6; i++) gp[6 * g + i] = 2 * G * (0.5 * eps[i] - pt.ep[i]);
    }
  }
  for (int a = 0; a < 8; a++)
    for (int c = 0; c < 6; c++) {
      double v = 0;
      for (int g = 0; g < 8; g++) v += G2N.M[a * 8 + g] * gp[6 * g + c];
      out[48 * (size_t)e + 6 * a + c] = (float)v;
    }
}

// _snapshot / _restore of the solder points' committed state (ep, s, ebar, W, sigEq)
__global__ void k_sub_points_copy(int np, const Point* __restrict__ from, Point* __restrict__ to) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= np) return;
  const Point& a = from[i];
  Point& b = to[i];
  for (int c = 0; c < 6; c++) b.ep[c] = a.ep[c];
  b.s = a.s; b.ebar = a.ebar; b.W = a.W; b.sigEq = a.sigEq;
}

// sampleLoop (13-fatigue.js:1032-1052) over one layer list: per entry the strain at the Gauss
// point (its own B-bar matrix), the stress at the committed plastic state (a 1e-9 s step) and
// the weighted shear stress and strain along the site's radial direction
__global__ void k_sub_sample(int cnt, const int* __restrict__ gp, const double* __restrict__ Bs, const int* __restrict__ conn,
                             const double* __restrict__ u, Point* __restrict__ pts, const int* __restrict__ eAn, AnandConst P,
                             const double* __restrict__ Etab, double T, double f, double cphi, double sphi, double* __restrict__ out) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= cnt) return;
  const int idx = gp[t], e = idx / 8, g = idx % 8;
  const double* Bb = Bs + 144 * (size_t)t;
  double ue[24], eps[6], sig[6];
  for (int a = 0; a < 8; a++) {
    const int n = conn[8 * (size_t)e + a];
    ue[3 * a] = u[3 * n]; ue[3 * a + 1] = u[3 * n + 1]; ue[3 * a + 2] = u[3 * n + 2];
  }
  for (int r = 0; r < 6; r++) {
    double s = 0;
    for (int c = 0; c < 24; c++) s += Bb[r * 24 + c] * ue[c];
    eps[r] = s;
  }
  eps[0] -= f; eps[1] -= f; eps[2] -= f;
  const StepK k = step_constants(P, Etab, T, 1e-9);
  anand_step(P, pts[8 * (size_t)eAn[e] + g], eps, k, sig, (double*)nullptr, false);
  out[2 * t] = sig[5] * cphi + sig[4] * sphi;
  out[2 * t + 1] = eps[5] * cphi + eps[4] * sphi;
}

// the layer averages of W and ebar (avg of run, :1020), in list order: one thread
__global__ void k_sub_layer_avg(int nDie, const int* __restrict__ dieGp, const double* __restrict__ dieW, int nSub,
                                const int* __restrict__ subGp, const double* __restrict__ subW, const Point* __restrict__ pts,
                                const int* __restrict__ eAn, double* __restrict__ out) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  for (int li = 0; li < 2; li++) {
    const int cnt = li == 0 ? nDie : nSub;
    const int* gp = li == 0 ? dieGp : subGp;
    const double* wv = li == 0 ? dieW : subW;
    double sW = 0, sE = 0, ws = 0;
    for (int q = 0; q < cnt; q++) {
      const int idx = gp[q];
      const Point& p = pts[8 * (size_t)eAn[idx / 8] + idx % 8];
      sW += wv[q] * p.W; sE += wv[q] * p.ebar; ws += wv[q];
    }
    out[2 * li] = ws != 0 ? sW / ws : CUDART_NAN;
    out[2 * li + 1] = ws != 0 ? sE / ws : CUDART_NAN;
  }
  // 0: W die, 1: ebar die, 2: W sub, 3: ebar sub
}

}  // namespace

// ---- the submodel ----------------------------------------------------------------------------------
struct SubModel {
  cudaStream_t st = nullptr;
  int nx = 0, ny = 0, nz = 0, nn = 0, ne = 0, ndof = 0, nbk = 0, nbnd = 0, nsolderE = 0;
  std::vector<double> xs, ys, zs, ts, solderE, solderF, ufE, ufF, siD, siF, subD, subF;
  double ufNu = 0, nuMax = 0, zt = 0, zaf = 0;
  AnandConst P{};
  int elasticSolder = 0;
  // homogenized-layer consistency mode: bump-layer solder fraction, global Poisson clamp, the top
  // substrate band's section (z ranges, stiffness and thermal strain tables per sub-layer)
  int uniform = 0, nsec = 0;
  double density = 0, nuMaxGlobal = 0.45;
  std::vector<double> secZ, secD, secF;
  // elastic material records: 4 materials, then (consistency mode) one per substrate element layer;
  // eRec is each element's record (d_eMat on the device)
  int nrec = 4;
  std::vector<int> conn, eIJK, eMat, eRec, eAn, rowPtr, col, diag, blkRow;
  std::vector<uint8_t> isC;
  int nglob = 0;
  // device
  DBuf<int> d_conn, d_eMat, d_eBb, d_eAn, d_rowPtr, d_col, d_diag, d_blkRow, d_blkStart, d_blkList, d_nodeStart, d_nodeList;
  DBuf<int> d_bNodes, d_bGlob;
  DBuf<uint8_t> d_isC;
  DBuf<double> d_Bm, d_Bw, d_bW, d_fields, d_u25, d_solderE, d_elas;
  DBuf<double> d_u, d_uN, d_sigE, d_eFn, d_eK, d_eF, d_fe, d_dmax, d_val, d_vals, d_s, d_rint, d_b, d_r, d_z, d_p, d_q, d_x, d_sums, d_pcg;
  DBuf<double> d_sumPart;               // the slices' partial sums (2 per slice)
  DBuf<Point> d_pts, d_snapPts;
  DBuf<double> d_snapU, d_snapSig, d_snapFn;
  DBuf<float> d_snapOut;                // a stress snapshot (48 per element)
  IcFactor ic;
  bool pcBuilt = false, pcStale = false;
  int pcIters = 0;
  // preconditioner of the inner solves: IC(0) as the reference, or the z-line block Jacobi
  int precond = TM_SUB_PC_IC;
  long long pcgSolves = 0, pcgIters = 0;   // inner solves and their PCG iterations so far
  DBuf<int> d_subBlk;                   // per node the block (n, n-1) of its column (-1 at the bottom)
  DBuf<double> d_lf;                    // z-line factors (LF_VALS per node)
  double Tn = 25;
  bool haveKey = false;
  double keyTn = 0, keyT = 0;
  // layer lists of run(): Gauss points (e*8 + g), volume weights, their own B-bar matrices
  std::vector<int> dieGp, subGp;
  std::vector<double> dieW, subW;
  DBuf<int> d_dieGp, d_subGp;
  DBuf<double> d_dieW, d_subW, d_dieB, d_subB, d_sample, d_avg;

  ~SubModel() {
    if (st) cudaStreamDestroy(st);
  }

  // the two sums of `kind` into out (device)
  void sums_dev(int n, int kind, const double* a, double* b, double* out) {
    note_launch(2);
    k_sub_sums_slice<<<sums_parts(n), SUMS_THREADS, 0, st>>>(n, kind, a, b, d_isC.p, d_sumPart.p);
    k_sub_sums_final<<<1, 32, 0, st>>>(n, d_sumPart.p, out);
    TM_CUDA_CHECK(cudaGetLastError());
  }
  void sums(int n, int kind, const double* a, double* b, double* h) {
    sums_dev(n, kind, a, b, d_sums.p);
    TM_CUDA_CHECK(cudaMemcpyAsync(h, d_sums.p, 2 * sizeof(double), cudaMemcpyDeviceToHost, st));
    TM_CUDA_CHECK(cudaStreamSynchronize(st));
  }

  // _elastic (13-fatigue.js:702-757); subZ: the element layer's mid-height for the substrate
  // slice in the consistency mode
  void elastic(int mat, double Ta, double Tb, double* D, double* sth, double subZ = 0) const {
    auto rowSum = [&](int r) { return D[r * 6] + D[r * 6 + 1] + D[r * 6 + 2]; };
    auto rowSumOf = [](const double* Dx, int r) { return Dx[r * 6] + Dx[r * 6 + 1] + Dx[r * 6 + 2]; };
    if (uniform && mat == M_UF) {
      // solder columns (columnD) and underfill superposed with volume fractions fb, 1 - fb
      double Es, Eu, Ds[36], Du[36];
      grid_mean(solderE.data(), 1, 1, Ta, Tb, &Es);
      grid_mean(ufE.data(), 1, 1, Ta, Tb, &Eu);
      column_d(Es, P.nu, Ds);
      iso_d(Eu, ufNu, nuMaxGlobal, Du);
      const double fs = grid_modulus_strain_increment(solderE.data(), solderF.data(), Ta, Tb) / Es;
      const double fu = grid_modulus_strain_increment(ufE.data(), ufF.data(), Ta, Tb) / Eu;
      for (int q = 0; q < 36; q++) D[q] = density * Ds[q] + (1 - density) * Du[q];
      for (int r = 0; r < 6; r++) sth[r] = density * rowSumOf(Ds, r) * fs + (1 - density) * rowSumOf(Du, r) * fu;
      return;
    }
    if (uniform && mat == M_SUB) {
      // the top band's own sub-layer stiffness at this height, with the through-thickness
      // response of the whole band: Voigt thickness modulus and Turner-weighted thermal strain
      const size_t DN = 36 * (size_t)TGRID_N, FN = 3 * (size_t)TGRID_N;
      int sl = nsec - 1;
      for (int q = 0; q < nsec; q++)
        if (subZ <= secZ[2 * q + 1] + 1e-12) { sl = q; break; }
      grid_mean(secD.data() + DN * sl, 36, 36, Ta, Tb, D);
      const double* Fsl = secF.data() + FN * sl;
      double dF[3];
      for (int c = 0; c < 2; c++) dF[c] = grid_at_s(Fsl, Tb, 3, c) - grid_at_s(Fsl, Ta, 3, c);
      double Ez = 0, EzF = 0, tt = 0, Dq[36], sq[6];
      for (int q = 0; q < nsec; q++) {
        const double tq = secZ[2 * q + 1] - secZ[2 * q];
        grid_mean(secD.data() + DN * q, 36, 36, Ta, Tb, Dq);
        const double* Fq = secF.data() + FN * q;
        const double fx = grid_at_s(Fq, Tb, 3, 0) - grid_at_s(Fq, Ta, 3, 0), fy = grid_at_s(Fq, Tb, 3, 1) - grid_at_s(Fq, Ta, 3, 1);
        grid_stress_increment(secD.data() + DN * q, Fq, Ta, Tb, sq);
        Ez += tq * Dq[14]; EzF += tq * (sq[2] - Dq[12] * fx - Dq[13] * fy); tt += tq;
      }
      D[14] = Ez / tt; dF[2] = EzF / Ez;
      for (int r = 0; r < 6; r++) sth[r] = D[r * 6] * dF[0] + D[r * 6 + 1] * dF[1] + D[r * 6 + 2] * dF[2];
      return;
    }
    auto isoStep = [&](const std::vector<double>& E, const std::vector<double>& F, double nu) {
      double Em;
      grid_mean(E.data(), 1, 1, Ta, Tb, &Em);
      const double ef = grid_modulus_strain_increment(E.data(), F.data(), Ta, Tb) / Em;
      iso_d(Em, nu, nuMax, D);
      for (int r = 0; r < 6; r++) sth[r] = rowSum(r) * ef;
    };
    if (mat == M_SI) {
      for (int q = 0; q < 36; q++) D[q] = siD[q];
      const double f = grid_at_s(siF.data(), Tb, 1, 0) - grid_at_s(siF.data(), Ta, 1, 0);
      for (int r = 0; r < 6; r++) sth[r] = rowSum(r) * f;
      return;
    }
    if (mat == M_UF) { isoStep(ufE, ufF, ufNu); return; }
    if (mat == M_SOLDER) { isoStep(solderE, solderF, P.nu); return; }
    grid_mean(subD.data(), 36, 36, Ta, Tb, D);
    grid_stress_increment(subD.data(), subF.data(), Ta, Tb, sth);
  }

  // fieldAt's two global temperatures around T and the blend between them
  void prescribe_args(double T, const double** fa, const double** fb, double* tOut) const {
    int i;
    const int n = (int)ts.size();
    if (T <= ts[0]) i = 0;
    else if (T >= ts[n - 1]) i = n - 2;
    else {
      int lo = 0, hi = n - 1;
      while (hi - lo > 1) { const int mid = (lo + hi) >> 1; if (ts[mid] <= T) lo = mid; else hi = mid; }
      i = lo;
    }
    double t = (T - ts[i]) / (ts[i + 1] - ts[i]);
    t = t < 0 ? 0 : (t > 1 ? 1 : t);
    const size_t G = 3 * (size_t)nglob;
    *fa = d_fields.p + G * i;
    *fb = d_fields.p + G * (i + 1);
    *tOut = t;
  }
  void prescribe(double T) {
    const double *fa, *fb;
    double t;
    prescribe_args(T, &fa, &fb, &t);
    note_launch();
    k_sub_prescribe<<<blocks_for(nbnd, 128), 128, 0, st>>>(nbnd, d_bNodes.p, d_bGlob.p, d_bW.p, fa, fb, t, d_u25.p, d_u.p);
    TM_CUDA_CHECK(cudaGetLastError());
  }

  // the solder's step constants at T over dt and its thermal strain from 25 degC
  void step_params(double T, double dt, StepK* kc, double* fSolder) const {
    const double E = grid_at_s(solderE.data(), T, 1, 0), nu = P.nu;
    const double expQ = std::exp(P.QR / (T + 273.15));
    *kc = StepK{E / (2 * (1 + nu)), E / (3 * (1 - 2 * nu)), expQ, dt * P.A / expQ, dt};
    *fSolder = grid_at_s(solderF.data(), T, 1, 0) - grid_at_s(solderF.data(), 25, 1, 0);
  }
  // whether the step from Tn to T needs its element matrices and material records built
  bool fresh_for(double T) const { return !(haveKey && keyTn == Tn && keyT == T); }

  // assemble (13-fatigue.js:776-853); returns the largest plastic increment
  double assemble(double T, double dt, bool wantK) {
    const bool fresh = fresh_for(T);
    if (fresh) upload_records(T);
    StepK kc;
    double fSolder;
    step_params(T, dt, &kc, &fSolder);
    note_launch(wantK ? 3 : 2);
    k_sub_assemble<<<blocks_for(ne, SA_WARPS), 32 * SA_WARPS, 0, st>>>(ne, d_conn.p, d_eMat.p, d_eBb.p, d_Bm.p, d_Bw.p, d_eAn.p, d_pts.p, d_u.p,
                                                                      d_uN.p, d_eFn.p, d_eK.p, d_eF.p, d_fe.p, d_dmax.p, d_elas.p, fresh,
                                                                      wantK, P, kc, fSolder);
    TM_CUDA_CHECK(cudaGetLastError());
    k_sub_gather_rint<<<blocks_for(ndof, 256), 256, 0, st>>>(ndof, d_nodeStart.p, d_nodeList.p, d_fe.p, d_rint.p);
    if (wantK)
      k_sub_gather_val<<<blocks_for(nbk, 128), 128, 0, st>>>(nbk, d_blkRow.p, d_col.p, d_blkStart.p, d_blkList.p, d_eK.p, d_isC.p, d_val.p);
    TM_CUDA_CHECK(cudaGetLastError());
    haveKey = true; keyTn = Tn; keyT = T;
    std::vector<double> dm(ne);
    d_dmax.download(dm.data(), ne, st);
    TM_CUDA_CHECK(cudaStreamSynchronize(st));
    double dMax = 0;
    for (int e = 0; e < ne; e++) if (dm[e] > dMax) dMax = dm[e];
    return dMax;
  }

  // _solve (13-fatigue.js:886-917): d_x = the Newton increment
  int solve(double tol) {
    note_launch(3);
    k_sub_scale_s<<<blocks_for(nn, 128), 128, 0, st>>>(nn, d_diag.p, d_val.p, d_s.p);
    k_sub_scale_vals<<<blocks_for(nbk, 128), 128, 0, st>>>(nbk, d_blkRow.p, d_col.p, d_s.p, d_val.p, d_vals.p);
    k_sub_rhs<<<blocks_for(ndof, 256), 256, 0, st>>>(ndof, d_rint.p, d_isC.p, d_s.p, d_b.p, d_r.p, d_x.p);
    TM_CUDA_CHECK(cudaGetLastError());
    if (precond == TM_SUB_PC_LINE) {
      note_launch();
      k_sub_line_factor<<<blocks_for((size_t)nx * ny, 128), 128, 0, st>>>(nx * ny, nz, d_diag.p, d_subBlk.p, d_vals.p, d_lf.p);
      TM_CUDA_CHECK(cudaGetLastError());
    } else if (!pcBuilt || pcStale) {
      ic_factor(ic, d_vals.p, st); pcBuilt = true; pcStale = false; pcIters = 0;
    }
    double h[2];
    sums(ndof, 1, d_b.p, d_b.p, h);
    const double bn = std::sqrt(h[0]);
    if (bn == 0) return 0;
    pc_apply(d_r.p, d_z.p);
    TM_CUDA_CHECK(cudaMemcpyAsync(d_p.p, d_z.p, ndof * sizeof(double), cudaMemcpyDeviceToDevice, st));
    // device scalars (k_sub_sums writes two values per result): rz at a, the next rz at 2 - a,
    // p.q at 4, r.r at 6; one host synchronization per iteration, for the convergence test
    double* S = d_pcg.p;
    int a = 0;
    sums_dev(ndof, 1, d_r.p, d_z.p, S + a);
    int it;
    const int nb = blocks_for(ndof, 256);
    double rr = 0;
    for (it = 1; it <= 2000; it++) {
      note_launch(2);
      k_sub_spmv<<<blocks_for(nn, 128), 128, 0, st>>>(nn, d_rowPtr.p, d_col.p, d_vals.p, d_p.p, d_q.p);
      sums_dev(ndof, 1, d_p.p, d_q.p, S + 4);
      k_sub_axpy2<<<nb, 256, 0, st>>>(ndof, S + a, S + 4, d_p.p, d_q.p, d_x.p, d_r.p);
      sums_dev(ndof, 1, d_r.p, d_r.p, S + 6);
      TM_CUDA_CHECK(cudaMemcpyAsync(&rr, S + 6, sizeof(double), cudaMemcpyDeviceToHost, st));
      TM_CUDA_CHECK(cudaStreamSynchronize(st));
      if (std::sqrt(rr) / bn < tol) break;
      pc_apply(d_r.p, d_z.p);
      note_launch();
      sums_dev(ndof, 1, d_r.p, d_z.p, S + (2 - a));
      k_sub_xpby<<<nb, 256, 0, st>>>(ndof, d_z.p, S + (2 - a), S + a, d_p.p);
      a = 2 - a;
    }
    TM_CUDA_CHECK(cudaGetLastError());
    note_launch();
    k_sub_mul<<<nb, 256, 0, st>>>(ndof, d_s.p, d_x.p);
    TM_CUDA_CHECK(cudaGetLastError());
    pcgSolves++;
    pcgIters += it;
    if (!pcIters) pcIters = it;
    else if (it > 2 * pcIters) pcStale = true;
    return it;
  }

  // z = M^-1 r with the submodel's preconditioner
  void pc_apply(const double* r, double* z) {
    if (precond == TM_SUB_PC_LINE) {
      note_launch();
      k_sub_line_apply<<<blocks_for((size_t)nx * ny, 128), 128, 0, st>>>(nx * ny, nz, d_lf.p, r, z);
      TM_CUDA_CHECK(cudaGetLastError());
    } else {
      ic_apply(ic, r, z, st);
    }
  }

  // the elastic material records of the step from Tn to T (_elasRec, 13-fatigue.js:760-773): the
  // 4 materials, then per substrate element layer in the consistency mode
  void fill_records(double T, double* h) const {
    for (int q = 0; q < 42 * nrec; q++) h[q] = 0;
    for (int m = 0; m < 4; m++) elastic(m, Tn, T, &h[42 * m], &h[42 * m + 36]);
    for (int k = 0; k + 4 < nrec; k++) elastic(M_SUB, Tn, T, &h[42 * (4 + k)], &h[42 * (4 + k) + 36], 0.5 * (zs[k] + zs[k + 1]));
  }
  void upload_records(double T) {
    std::vector<double> h(42 * (size_t)nrec, 0.0);
    fill_records(T, h.data());
    d_elas.upload(h, st);
  }

  void commit_elastic(double T) {
    // the step's material records are those of the assembly from Tn to T
    if (!(haveKey && keyTn == Tn && keyT == T)) upload_records(T);
    note_launch();
    k_sub_commit_elastic<<<blocks_for(ne, SA_WARPS), 32 * SA_WARPS, 0, st>>>(ne, d_conn.p, d_eMat.p, d_eBb.p, d_Bm.p, d_Bw.p, d_eAn.p, d_u.p,
                                                                            d_uN.p, d_elas.p, d_sigE.p, d_eFn.p);
    TM_CUDA_CHECK(cudaGetLastError());
    TM_CUDA_CHECK(cudaMemcpyAsync(d_uN.p, d_u.p, ndof * sizeof(double), cudaMemcpyDeviceToDevice, st));
    Tn = T;
  }

  // stepTo (13-fatigue.js:924-956)
  bool step_to(double T, double dt, int* newton, double* dMaxOut) {
    prescribe(T);
    double dMax = 0, rPrev = INFINITY;
    bool converged = false, haveK = false;
    int it;
    double h[2];
    for (it = 1; it <= SUB_NEWTON_MAXIT; it++) {
      const bool wantK = it <= 2 || !haveK;
      dMax = assemble(T, dt, wantK);
      if (wantK) haveK = true;
      sums(ndof, 0, d_rint.p, nullptr, h);
      const double rn = std::sqrt(h[0]), fn = std::sqrt(h[1]);
      const double ref = std::max(fn, 1e-30);
      if (rn / ref < SUB_RES_TOL) { converged = true; break; }
      if (!wantK && rn > 0.5 * rPrev) assemble(T, dt, true);   // stalled with the frozen tangent: refresh it
      rPrev = rn;
      solve(std::max(SUB_INNER_TOL, std::min(1e-3, 0.01 * SUB_RES_TOL * ref / std::max(rn, 1e-300))));
      sums(ndof, 2, d_x.p, d_u.p, h);   // u += du on the free DOFs
      if (std::sqrt(h[0]) < SUB_DU_TOL * std::max(std::sqrt(h[1]), 1e-30)) { converged = true; it++; break; }
    }
    if (converged) {
      dMax = assemble(T, dt, false);
      if (nsolderE) {
        note_launch();
        k_sub_commit_points<<<blocks_for(8 * (size_t)nsolderE, 128), 128, 0, st>>>(8 * nsolderE, d_pts.p);
        TM_CUDA_CHECK(cudaGetLastError());
      }
      commit_elastic(T);
    }
    *newton = it; *dMaxOut = dMax;
    TM_CUDA_CHECK(cudaStreamSynchronize(st));
    return converged;
  }

  void snapshot() {
    TM_CUDA_CHECK(cudaMemcpyAsync(d_snapU.p, d_u.p, ndof * sizeof(double), cudaMemcpyDeviceToDevice, st));
    TM_CUDA_CHECK(cudaMemcpyAsync(d_snapSig.p, d_sigE.p, 48 * (size_t)ne * sizeof(double), cudaMemcpyDeviceToDevice, st));
    TM_CUDA_CHECK(cudaMemcpyAsync(d_snapFn.p, d_eFn.p, 24 * (size_t)ne * sizeof(double), cudaMemcpyDeviceToDevice, st));
    if (nsolderE) {
      note_launch();
      k_sub_points_copy<<<blocks_for(8 * (size_t)nsolderE, 128), 128, 0, st>>>(8 * nsolderE, d_pts.p, d_snapPts.p);
    }
  }
  void restore(double snapTn) {
    TM_CUDA_CHECK(cudaMemcpyAsync(d_u.p, d_snapU.p, ndof * sizeof(double), cudaMemcpyDeviceToDevice, st));
    TM_CUDA_CHECK(cudaMemcpyAsync(d_uN.p, d_snapU.p, ndof * sizeof(double), cudaMemcpyDeviceToDevice, st));
    TM_CUDA_CHECK(cudaMemcpyAsync(d_sigE.p, d_snapSig.p, 48 * (size_t)ne * sizeof(double), cudaMemcpyDeviceToDevice, st));
    TM_CUDA_CHECK(cudaMemcpyAsync(d_eFn.p, d_snapFn.p, 24 * (size_t)ne * sizeof(double), cudaMemcpyDeviceToDevice, st));
    if (nsolderE) {
      note_launch();
      k_sub_points_copy<<<blocks_for(8 * (size_t)nsolderE, 128), 128, 0, st>>>(8 * nsolderE, d_snapPts.p, d_pts.p);
    }
    Tn = snapTn;
  }

  // sampleLoop: the two lists in order (a point in both is stepped twice, as in the reference)
  void sample_loop(double T, double cphi, double sphi, double* L) {
    const double f = grid_at_s(solderF.data(), T, 1, 0) - grid_at_s(solderF.data(), 25, 1, 0);
    double s[6] = {0, 0, 0, 0, 0, 0};   // tS, gS, wS, tB, gB, wB
    for (int li = 0; li < 2; li++) {
      const int cnt = li == 0 ? (int)dieGp.size() : (int)subGp.size();
      if (!cnt) continue;
      note_launch();
      k_sub_sample<<<blocks_for(cnt, 64), 64, 0, st>>>(cnt, li == 0 ? d_dieGp.p : d_subGp.p, li == 0 ? d_dieB.p : d_subB.p, d_conn.p, d_u.p,
                                                      d_pts.p, d_eAn.p, P, d_solderE.p, T, f, cphi, sphi, d_sample.p);
      TM_CUDA_CHECK(cudaGetLastError());
      std::vector<double> o(2 * (size_t)cnt);
      d_sample.download(o.data(), o.size(), st);
      TM_CUDA_CHECK(cudaStreamSynchronize(st));
      const std::vector<double>& wv = li == 0 ? dieW : subW;
      for (int q = 0; q < cnt; q++) {
        s[3 * li] += wv[q] * o[2 * q]; s[3 * li + 1] += wv[q] * o[2 * q + 1]; s[3 * li + 2] += wv[q];
      }
    }
    L[0] = s[2] != 0 ? s[0] / s[2] : NAN; L[1] = s[2] != 0 ? s[1] / s[2] : NAN;
    L[2] = s[5] != 0 ? s[3] / s[5] : NAN; L[3] = s[5] != 0 ? s[4] / s[5] : NAN;
  }

  // W and ebar averaged over the two interface layers (avg of run, 13-fatigue.js:1020): die W, die
  // ebar, substrate W, substrate ebar
  void layer_avg(double* avg) {
    note_launch();
    k_sub_layer_avg<<<1, 1, 0, st>>>((int)dieGp.size(), d_dieGp.p, d_dieW.p, (int)subGp.size(), d_subGp.p, d_subW.p, d_pts.p, d_eAn.p,
                                    d_avg.p);
    TM_CUDA_CHECK(cudaGetLastError());
    d_avg.download(avg, 4, st);
    TM_CUDA_CHECK(cudaStreamSynchronize(st));
  }

  // _stressSnapshot at temperature T into host memory (48 floats per element)
  void stress_snapshot(double T, float* host) {
    GpToNode G2N;
    const double s3 = std::sqrt(3.0);
    for (int n = 0; n < 8; n++) {
      const double xi = HX[n] * s3, eta = HY[n] * s3, zeta = HZ[n] * s3;
      for (int g = 0; g < 8; g++) G2N.M[n * 8 + g] = 0.125 * (1 + HX[g] * xi) * (1 + HY[g] * eta) * (1 + HZ[g] * zeta);
    }
    const double E = grid_at_s(solderE.data(), T, 1, 0);
    const double f = grid_at_s(solderF.data(), T, 1, 0) - grid_at_s(solderF.data(), 25, 1, 0);
    d_snapOut.alloc(48 * (size_t)ne);
    note_launch();
    k_sub_stress_snapshot<<<blocks_for(ne, 128), 128, 0, st>>>(ne, d_conn.p, d_eAn.p, d_eBb.p, d_Bm.p, d_pts.p, d_u.p, d_sigE.p, E, P.nu, f,
                                                              G2N, d_snapOut.p);
    TM_CUDA_CHECK(cudaGetLastError());
    TM_CUDA_CHECK(cudaMemcpyAsync(host, d_snapOut.p, 48 * (size_t)ne * sizeof(float), cudaMemcpyDeviceToHost, st));
    TM_CUDA_CHECK(cudaStreamSynchronize(st));
  }

  // run; with hphase, the stress snapshots at the end of each ramp and dwell of the last cycle
  // (13-fatigue.js:1053-1078): *nSnaps of them, up to maxSnaps written (meta: T, t, cycle, phase)
  void run(int nsteps, const double* ht, const double* hT, const int* hcycle, int cycles, double cphi, double sphi, double* out,
           double* perCycle, double* loop, const int* hphase = nullptr, int maxSnaps = 0, int* nSnaps = nullptr, double* snapMeta = nullptr,
           float* snapSig = nullptr) {
    if (!nsolderE || elasticSolder) fail(TM_BAD_INPUT, "submodel run needs Anand solder points");
    if (nSnaps) *nSnaps = 0;
    std::vector<double> Wdie(cycles + 1, 0.0), Wsub(cycles + 1, 0.0), Edie(cycles + 1, 0.0), Esub(cycles + 1, 0.0);
    long long totalNewton = 0;
    int cutbacks = 0, steps = 0, nsubNext = 1, sample = 0;
    sample_loop(25, cphi, sphi, loop + 4 * (size_t)sample++);
    double avg[4];
    for (int k = 1; k < nsteps; k++) {
      const double T0 = hT[k - 1], T1 = hT[k], t0s = ht[k - 1], t1s = ht[k];
      int nsub = nsubNext;
      bool done = false;
      double dLast = 0;
      for (int attempt = 0; attempt < 8 && !done; attempt++) {
        const double snapTn = Tn;
        snapshot();
        bool ok = true;
        for (int s = 1; s <= nsub; s++) {
          const double T = T0 + (T1 - T0) * s / nsub, dt = (t1s - t0s) / nsub;
          int newton;
          double dMax;
          const bool conv = step_to(T, dt, &newton, &dMax);
          totalNewton += newton;
          steps++;
          dLast = dMax;
          if (!conv || dMax > INELASTIC_STEP_MAX) { ok = false; break; }
        }
        if (ok) done = true;
        else { restore(snapTn); nsub *= 2; cutbacks++; }
      }
      nsubNext = dLast > 0.5 * INELASTIC_STEP_MAX ? std::min(nsub * 2, 64) : (dLast < 0.2 * INELASTIC_STEP_MAX ? std::max(1, nsub >> 1) : nsub);
      if (!done) fail(TM_NOT_CONVERGED, "submodel step failed to converge after cutbacks");
      sample_loop(T1, cphi, sphi, loop + 4 * (size_t)sample++);
      layer_avg(avg);
      const int c = hcycle[k];
      if (hphase && nSnaps && c == cycles && (k == nsteps - 1 || hphase[k + 1] != hphase[k])) {
        const int q = (*nSnaps)++;
        if (q < maxSnaps) {
          double* mt = snapMeta + 4 * (size_t)q;
          mt[0] = T1; mt[1] = t1s; mt[2] = c; mt[3] = hphase[k];
          stress_snapshot(T1, snapSig + 48 * (size_t)ne * q);
        }
      }
      Wdie[c] = avg[0]; Edie[c] = avg[1]; Wsub[c] = avg[2]; Esub[c] = avg[3];
    }
    const int nc = cycles;
    const double dWdie = Wdie[nc] - Wdie[nc - 1], dWsub = Wsub[nc] - Wsub[nc - 1];
    const double dEdie = Edie[nc] - Edie[nc - 1], dEsub = Esub[nc] - Esub[nc - 1];
    const double dW = std::max(dWdie, dWsub), dE = dWdie >= dWsub ? dEdie : dEsub;
    const double prev = nc >= 2 ? std::max(Wdie[nc - 1] - Wdie[nc - 2], Wsub[nc - 1] - Wsub[nc - 2]) : NAN;
    const double stab = std::isfinite(prev) && prev > 0 ? std::fabs(dW - prev) / prev : NAN;
    const double o[10] = {dW, dWdie, dWsub, dE, dEdie, dEsub, stab, (double)steps, (double)cutbacks, (double)totalNewton / std::max(steps, 1)};
    std::copy(o, o + 10, out);
    for (int c = 1; c <= nc; c++) { perCycle[2 * (c - 1)] = Wdie[c] - Wdie[c - 1]; perCycle[2 * (c - 1) + 1] = Wsub[c] - Wsub[c - 1]; }
  }
};

SubModel* submodel_create(const tm_submodel_spec& sp) {
  if (sp.nx < 2 || sp.ny < 2 || sp.nz < 2 || !sp.xs || !sp.ys || !sp.zs || !sp.cellMat || sp.nt < 2 || !sp.ts || !sp.fields ||
      !sp.u25 || !sp.bGlob || !sp.bW || !sp.solder.Etab || !sp.solder.Ftab || !sp.ufE || !sp.ufF || !sp.siD || !sp.siF || !sp.subD ||
      !sp.subF || sp.nglob < 1)
    fail(TM_BAD_INPUT, "submodel: missing input");
  std::unique_ptr<SubModel> S(new SubModel());
  SubModel& m = *S;
  TM_CUDA_CHECK(cudaStreamCreateWithFlags(&m.st, cudaStreamNonBlocking));
  m.nx = sp.nx; m.ny = sp.ny; m.nz = sp.nz;
  m.xs.assign(sp.xs, sp.xs + sp.nx); m.ys.assign(sp.ys, sp.ys + sp.ny); m.zs.assign(sp.zs, sp.zs + sp.nz);
  m.ts.assign(sp.ts, sp.ts + sp.nt);
  m.solderE.assign(sp.solder.Etab, sp.solder.Etab + TGRID_N); m.solderF.assign(sp.solder.Ftab, sp.solder.Ftab + TGRID_N);
  m.ufE.assign(sp.ufE, sp.ufE + TGRID_N); m.ufF.assign(sp.ufF, sp.ufF + TGRID_N);
  m.siD.assign(sp.siD, sp.siD + 36); m.siF.assign(sp.siF, sp.siF + TGRID_N);
  m.subD.assign(sp.subD, sp.subD + 36 * TGRID_N); m.subF.assign(sp.subF, sp.subF + 3 * TGRID_N);
  m.ufNu = sp.ufNu; m.nuMax = sp.nuMax; m.zt = sp.zt; m.zaf = sp.zaf;
  if (sp.uniformMaterial) {
    if (sp.nsec < 1 || !sp.secZ || !sp.secD || !sp.secF) fail(TM_BAD_INPUT, "submodel: the consistency mode needs the band section");
    if (!(sp.density >= 0 && sp.density <= 1)) fail(TM_BAD_INPUT, "submodel: bump density outside [0, 1]");
    m.uniform = 1;
    m.density = sp.density;
    m.nuMaxGlobal = sp.nuMaxGlobal;
    m.nsec = sp.nsec;
    m.secZ.assign(sp.secZ, sp.secZ + 2 * (size_t)sp.nsec);
    m.secD.assign(sp.secD, sp.secD + 36 * (size_t)TGRID_N * sp.nsec);
    m.secF.assign(sp.secF, sp.secF + 3 * (size_t)TGRID_N * sp.nsec);
    m.nrec = 4 + (sp.nz - 1);
  }
  m.P = AnandConst{sp.solder.A, sp.solder.QR, sp.solder.xi, sp.solder.m, sp.solder.shat, sp.solder.n, sp.solder.h0, sp.solder.a,
                   sp.solder.s0, sp.solder.nu};
  m.elasticSolder = sp.elasticSolder;
  m.nglob = sp.nglob;
  const int nx = m.nx, ny = m.ny, nz = m.nz, ncy = ny - 1, ncz = nz - 1;
  // every cell holds one element: nodes (i ny + j) nz + k, elements in cell order (06-mesher.js:14-72)
  m.nn = nx * ny * nz;
  m.ne = (nx - 1) * ncy * ncz;
  m.ndof = 3 * m.nn;
  const int LOC[8][3] = {{0, 0, 0}, {1, 0, 0}, {1, 1, 0}, {0, 1, 0}, {0, 0, 1}, {1, 0, 1}, {1, 1, 1}, {0, 1, 1}};
  m.conn.resize(8 * (size_t)m.ne); m.eIJK.resize(3 * (size_t)m.ne); m.eMat.resize(m.ne); m.eRec.resize(m.ne); m.eAn.assign(m.ne, -1);
  for (int i = 0, e = 0; i < nx - 1; i++)
    for (int j = 0; j < ncy; j++)
      for (int k = 0; k < ncz; k++, e++) {
        int mat = sp.cellMat[e];
        if (mat < 0 || mat > 3) fail(TM_BAD_INPUT, "submodel: cell material out of range");
        if (m.uniform && mat == M_SOLDER) mat = M_UF;   // the bump layer's phases homogenized (13-fatigue.js:538)
        m.eMat[e] = mat;
        m.eRec[e] = m.uniform && mat == M_SUB ? 4 + k : mat;
        m.eIJK[3 * e] = i; m.eIJK[3 * e + 1] = j; m.eIJK[3 * e + 2] = k;
        for (int a = 0; a < 8; a++) m.conn[8 * (size_t)e + a] = ((i + LOC[a][0]) * ny + j + LOC[a][1]) * nz + k + LOC[a][2];
        if (mat == M_SOLDER && !m.elasticSolder) m.eAn[e] = m.nsolderE++;
      }
  // full block pattern (nodes sharing an element: the 27-point neighbourhood), sorted
  m.rowPtr.assign(m.nn + 1, 0);
  for (int i = 0; i < nx; i++)
    for (int j = 0; j < ny; j++)
      for (int k = 0; k < nz; k++) {
        const int n = (i * ny + j) * nz + k;
        for (int di = -1; di <= 1; di++)
          for (int dj = -1; dj <= 1; dj++)
            for (int dk = -1; dk <= 1; dk++) {
              const int a = i + di, b = j + dj, c = k + dk;
              if (a < 0 || b < 0 || c < 0 || a >= nx || b >= ny || c >= nz) continue;
              m.col.push_back((a * ny + b) * nz + c);
              m.blkRow.push_back(n);
            }
        m.rowPtr[n + 1] = (int)m.col.size();
      }
  m.nbk = (int)m.col.size();
  m.diag.assign(m.nn, 0);
  for (int n = 0; n < m.nn; n++)
    for (int k = m.rowPtr[n]; k < m.rowPtr[n + 1]; k++) if (m.col[k] == n) { m.diag[n] = k; break; }
  // gather lists: per block the (e, a, b) contributions and per node the (e, a), in element order
  std::vector<int> bcnt(m.nbk + 1, 0), ncnt(m.nn + 1, 0), bmap(64 * (size_t)m.ne);
  for (int e = 0; e < m.ne; e++)
    for (int a = 0; a < 8; a++) {
      const int na = m.conn[8 * (size_t)e + a];
      ncnt[na + 1]++;
      for (int b = 0; b < 8; b++) {
        const int nb = m.conn[8 * (size_t)e + b];
        const int k = (int)(std::lower_bound(m.col.begin() + m.rowPtr[na], m.col.begin() + m.rowPtr[na + 1], nb) - m.col.begin());
        bmap[64 * (size_t)e + 8 * a + b] = k;
        bcnt[k + 1]++;
      }
    }
  for (int k = 0; k < m.nbk; k++) bcnt[k + 1] += bcnt[k];
  for (int n = 0; n < m.nn; n++) ncnt[n + 1] += ncnt[n];
  std::vector<int> blist(bcnt[m.nbk]), nlist(ncnt[m.nn]);
  {
    std::vector<int> bf(bcnt.begin(), bcnt.end() - 1), nf(ncnt.begin(), ncnt.end() - 1);
    for (int e = 0; e < m.ne; e++)
      for (int a = 0; a < 8; a++) {
        nlist[nf[m.conn[8 * (size_t)e + a]]++] = 8 * e + a;
        for (int b = 0; b < 8; b++) { const int k = bmap[64 * (size_t)e + 8 * a + b]; blist[bf[k]++] = 64 * e + 8 * a + b; }
      }
  }
  if ((long long)m.ne * 64 >= (1LL << 31)) fail(TM_BAD_INPUT, "submodel too large");
  // boundary: nodes on the six faces, ascending
  m.isC.assign(m.ndof, 0);
  std::vector<int> bNodes;
  for (int i = 0; i < nx; i++)
    for (int j = 0; j < ny; j++)
      for (int k = 0; k < nz; k++)
        if (i == 0 || j == 0 || k == 0 || i == nx - 1 || j == ny - 1 || k == nz - 1) {
          const int n = (i * ny + j) * nz + k;
          bNodes.push_back(n);
          m.isC[3 * n] = m.isC[3 * n + 1] = m.isC[3 * n + 2] = 1;
        }
  std::sort(bNodes.begin(), bNodes.end());
  if ((int)bNodes.size() != sp.nb) fail(TM_BAD_INPUT, "submodel: boundary node count does not match the cell");
  m.nbnd = sp.nb;
  for (int q = 0; q < 8 * sp.nb; q++)
    if (sp.bGlob[q] < 0 || sp.bGlob[q] >= sp.nglob) fail(TM_BAD_INPUT, "submodel: boundary global node out of range");
  // _bbarCache: the 8 Gauss-point B-bar matrices per distinct element size (12 significant digits)
  std::map<std::string, int> keys;
  std::vector<int> eBb(m.ne);
  std::vector<double> Bm, Bw;
  const double GP = 1 / std::sqrt(3.0);
  for (int e = 0; e < m.ne; e++) {
    const int i = m.eIJK[3 * e], j = m.eIJK[3 * e + 1], k = m.eIJK[3 * e + 2];
    const double hx = m.xs[i + 1] - m.xs[i], hy = m.ys[j + 1] - m.ys[j], hz = m.zs[k + 1] - m.zs[k];
    char buf[96];
    snprintf(buf, sizeof buf, "%.11e|%.11e|%.11e", hx, hy, hz);
    auto it = keys.find(buf);
    if (it != keys.end()) { eBb[e] = it->second; continue; }
    const int idx = (int)Bw.size();
    keys.emplace(buf, idx);
    Bm.resize(Bm.size() + 8 * 144);
    for (int g = 0; g < 8; g++) bbar_matrix(hx, hy, hz, HX[g] * GP, HY[g] * GP, HZ[g] * GP, Bm.data() + (size_t)idx * 8 * 144 + 144 * g);
    Bw.push_back(hx * hy * hz / 8);
    eBb[e] = idx;
  }
  // layer lists of run(): solder Gauss points in the averaging layers, with their own B-bar matrices
  std::vector<double> dieB, subB;
  for (int e = 0; e < m.ne; e++) {
    if (m.eMat[e] != M_SOLDER) continue;
    const int i = m.eIJK[3 * e], j = m.eIJK[3 * e + 1], k = m.eIJK[3 * e + 2];
    const double zc = 0.5 * (m.zs[k] + m.zs[k + 1]);
    const double hx = m.xs[i + 1] - m.xs[i], hy = m.ys[j + 1] - m.ys[j], hz = m.zs[k + 1] - m.zs[k];
    const double w = hx * hy * hz / 8;
    for (int g = 0; g < 8; g++) {
      double B[144];
      bbar_matrix(hx, hy, hz, HX[g] * GP, HY[g] * GP, HZ[g] * GP, B);
      if (zc > m.zaf - SUB_T_AVG) { m.dieGp.push_back(8 * e + g); m.dieW.push_back(w); dieB.insert(dieB.end(), B, B + 144); }
      if (zc < m.zt + SUB_T_AVG) { m.subGp.push_back(8 * e + g); m.subW.push_back(w); subB.insert(subB.end(), B, B + 144); }
    }
  }
  // device copies and state
  cudaStream_t st = m.st;
  m.d_conn.upload(m.conn, st); m.d_eMat.upload(m.eRec, st); m.d_eBb.upload(eBb, st); m.d_eAn.upload(m.eAn, st);
  m.d_rowPtr.upload(m.rowPtr, st); m.d_col.upload(m.col, st); m.d_diag.upload(m.diag, st); m.d_blkRow.upload(m.blkRow, st);
  m.d_blkStart.upload(bcnt, st); m.d_blkList.upload(blist, st); m.d_nodeStart.upload(ncnt, st); m.d_nodeList.upload(nlist, st);
  m.d_bNodes.upload(bNodes, st); m.d_bGlob.upload(sp.bGlob, 8 * (size_t)sp.nb, st); m.d_bW.upload(sp.bW, 8 * (size_t)sp.nb, st);
  m.d_isC.upload(m.isC, st);
  m.d_Bm.upload(Bm, st); m.d_Bw.upload(Bw, st);
  m.d_fields.upload(sp.fields, (size_t)sp.nt * sp.nglob * 3, st); m.d_u25.upload(sp.u25, 3 * (size_t)sp.nglob, st);
  m.d_solderE.upload(m.solderE, st);
  m.d_elas.alloc(4 * 42);
  const size_t n = m.ndof;
  for (DBuf<double>* b : {&m.d_u, &m.d_uN, &m.d_rint, &m.d_b, &m.d_r, &m.d_z, &m.d_p, &m.d_q, &m.d_x, &m.d_s, &m.d_snapU}) { b->alloc(n); b->zero(st); }
  m.d_sigE.alloc(48 * (size_t)m.ne); m.d_sigE.zero(st);
  m.d_eFn.alloc(24 * (size_t)m.ne); m.d_eFn.zero(st);
  m.d_snapSig.alloc(48 * (size_t)m.ne); m.d_snapFn.alloc(24 * (size_t)m.ne);
  m.d_eK.alloc(576 * (size_t)m.ne); m.d_eF.alloc(24 * (size_t)m.ne); m.d_fe.alloc(24 * (size_t)m.ne); m.d_dmax.alloc(m.ne);
  m.d_val.alloc(9 * (size_t)m.nbk); m.d_vals.alloc(9 * (size_t)m.nbk);
  m.d_sums.alloc(2); m.d_avg.alloc(4); m.d_pcg.alloc(8); m.d_sumPart.alloc(2 * SUMS_MAXP);
  if (m.nsolderE) {
    std::vector<Point> pts(8 * (size_t)m.nsolderE);
    for (Point& p : pts) {
      for (int c = 0; c < 6; c++) { p.ep[c] = 0; p.tr_ep[c] = 0; }
      p.s = m.P.s0; p.ebar = 0; p.W = 0; p.sigEq = 0; p.lastD = 0;
      p.tr_s = 0; p.tr_ebar = 0; p.tr_W = 0; p.tr_sigEq = 0;
    }
    m.d_pts.upload(pts, st);
    m.d_snapPts.alloc(pts.size());
  }
  m.d_dieGp.upload(m.dieGp, st); m.d_subGp.upload(m.subGp, st); m.d_dieW.upload(m.dieW, st); m.d_subW.upload(m.subW, st);
  m.d_dieB.upload(dieB, st); m.d_subB.upload(subB, st);
  m.d_sample.alloc(2 * std::max(m.dieGp.size(), m.subGp.size()) + 2);
  // the z-line preconditioner's column couplings
  std::vector<int> subBlk(m.nn, -1);
  for (int n = 0; n < m.nn; n++)
    if (n % nz)
      for (int k = m.rowPtr[n]; k < m.rowPtr[n + 1]; k++) if (m.col[k] == n - 1) { subBlk[n] = k; break; }
  m.d_subBlk.upload(subBlk, st);
  m.d_lf.alloc((size_t)LF_VALS * m.nn);
  // IC(0) structure of the tangent's pattern (values at 9k + 3p + q)
  std::vector<long long> vbase(m.nbk);
  for (int k = 0; k < m.nbk; k++) vbase[k] = 9LL * k;
  ic_build_structure(m.ic, m.nn, m.rowPtr, m.col, vbase, 1, st);
  TM_CUDA_CHECK(cudaStreamSynchronize(st));
  return S.release();
}

void submodel_destroy(SubModel* s) { delete s; }

bool submodel_step(SubModel& s, double T, double dt, int* newton, double* dMax) { return s.step_to(T, dt, newton, dMax); }

void submodel_get(SubModel& s, double* u, double* W, double* ebar) {
  if (u) { s.d_u.download(u, s.ndof, s.st); }
  if ((W || ebar) && s.nsolderE) {
    std::vector<Point> pts(8 * (size_t)s.nsolderE);
    s.d_pts.download(pts.data(), pts.size(), s.st);
    TM_CUDA_CHECK(cudaStreamSynchronize(s.st));
    for (size_t q = 0; q < pts.size(); q++) { if (W) W[q] = pts[q].W; if (ebar) ebar[q] = pts[q].ebar; }
  }
  TM_CUDA_CHECK(cudaStreamSynchronize(s.st));
}

void submodel_sizes(SubModel& s, int64_t* out) {
  out[0] = s.nn; out[1] = s.ne; out[2] = s.nbnd; out[3] = 8LL * s.nsolderE;
}

void submodel_counters(SubModel& s, int64_t* out) {
  out[0] = s.pcgSolves; out[1] = s.pcgIters;
}

void submodel_run(SubModel& s, int nsteps, const double* t, const double* T, const int* cycle, int cycles, double cphi, double sphi,
                  double* out, double* perCycle, double* loop, const int* phase, int maxSnaps, int* nSnaps, double* snapMeta,
                  float* snapSig) {
  if (nsteps < 2 || cycles < 1) fail(TM_BAD_INPUT, "submodel run: need >= 2 history points and >= 1 cycle");
  for (int k = 0; k < nsteps; k++) if (cycle[k] < 0 || cycle[k] > cycles) fail(TM_BAD_INPUT, "submodel run: cycle index out of range");
  if (maxSnaps > 0 && (!snapMeta || !snapSig)) fail(TM_BAD_INPUT, "submodel run: snapshot buffers missing");
  s.run(nsteps, t, T, cycle, cycles, cphi, sphi, out, perCycle, loop, phase, maxSnaps, nSnaps, snapMeta, snapSig);
}

void submodel_stress_snapshot(SubModel& s, double T, float* out) { s.stress_snapshot(T, out); }

void submodel_set_precond(SubModel& s, int kind) {
  if (kind != TM_SUB_PC_IC && kind != TM_SUB_PC_LINE) fail(TM_BAD_INPUT, "submodel: unknown preconditioner kind");
  s.precond = kind;
  s.pcBuilt = false;
}


// ---- batched submodels ------------------------------------------------------------------------------
// Submodels over the same cycle history advance together: each phase of their Newton steps
// (prescription, assembly and gathers, residual norms, the inner PCG's products, updates,
// preconditioner and reductions, commits) is one launch over every submodel in that phase, its
// CTAs mapped to (submodel, block of items) through a segment table passed by value. Every
// submodel keeps its own sub-step, cutback and Newton state on the host (run(), 13-fatigue.js:
// 1004-1104, stepTo :924-956) and takes exactly the operations of the single engine, so with the
// same preconditioner a batched submodel's result is the single engine's bit for bit.
namespace {

constexpr int SB_MAX = 64;   // submodels per batch

// one submodel's device arrays as the batched kernels read them
struct SubView {
  int ne, nn, ndof, nbk, nbnd, ncol, nz, npts;
  const int *conn, *eMat, *eBb, *eAn, *rowPtr, *col, *diag, *blkRow, *blkStart, *blkList, *nodeStart, *nodeList, *bNodes, *bGlob, *subBlk;
  const uint8_t* isC;
  const double *Bm, *Bw, *bW, *u25, *elas;
  double *u, *uN, *sigE, *eFn, *eK, *eF, *fe, *dmax, *val, *vals, *s, *rint, *b, *r, *z, *p, *q, *x, *lf, *sumPart;
  Point* pts;
};
// one submodel's parameters of the current phase
struct SubRound {
  AnandConst P;
  StepK kc;
  double fSolder, t;
  const double *fa, *fb;
  int fresh, wantK;
};
// the submodels of one launch and the first CTA of each
struct Seg {
  int n;
  int sub[SB_MAX];
  int start[SB_MAX + 1];
};

__device__ __forceinline__ int seg_find(const Seg& g, int blk) {
  int lo = 0, hi = g.n - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (g.start[mid] <= blk) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}
// the CTA's submodel and the index of its thread's item (items of `per` per CTA, one per thread)
#define SB_ITEM(per)                                              \
  const int sq_ = seg_find(g, blockIdx.x);                        \
  const int sub = g.sub[sq_];                                     \
  const SubView& v = V[sub];                                      \
  const int item = (blockIdx.x - g.start[sq_]) * (per) + threadIdx.x

__global__ void kb_prescribe(Seg g, const SubView* __restrict__ V, const SubRound* __restrict__ R) {
  SB_ITEM(blockDim.x);
  if (item < v.nbnd) sub_prescribe_node(item, v.bNodes, v.bGlob, v.bW, R[sub].fa, R[sub].fb, R[sub].t, v.u25, v.u);
}
__global__ void __launch_bounds__(32 * SA_WARPS) kb_assemble(Seg g, const SubView* __restrict__ V, const SubRound* __restrict__ R) {
  __shared__ AsmSmem sm[SA_WARPS];
  const int sq = seg_find(g, blockIdx.x), sub = g.sub[sq];
  const SubView& v = V[sub];
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int e = (blockIdx.x - g.start[sq]) * SA_WARPS + w;
  if (e >= v.ne) return;
  const SubRound& r = R[sub];
  sub_assemble_element(e, lane, sm[w], v.conn, v.eMat, v.eBb, v.Bm, v.Bw, v.eAn, v.pts, v.u, v.uN, v.eFn, v.eK, v.eF, v.fe, v.dmax, v.elas,
                       r.fresh, r.wantK, r.P, r.kc, r.fSolder);
}
__global__ void kb_gather_rint(Seg g, const SubView* __restrict__ V) {
  SB_ITEM(blockDim.x);
  if (item < v.ndof) sub_gather_rint_dof(item, v.nodeStart, v.nodeList, v.fe, v.rint);
}
__global__ void kb_gather_val(Seg g, const SubView* __restrict__ V) {
  SB_ITEM(blockDim.x);
  if (item < v.nbk) sub_gather_val_block(item, v.blkRow, v.col, v.blkStart, v.blkList, v.eK, v.isC, v.val);
}
// the largest plastic increment of each submodel (CTA per submodel)
__global__ void __launch_bounds__(256) kb_dmax(Seg g, const SubView* __restrict__ V, double* __restrict__ out) {
  __shared__ double red[256];
  const int sub = g.sub[blockIdx.x];
  const SubView& v = V[sub];
  double m = 0;
  for (int e = threadIdx.x; e < v.ne; e += 256) {
    const double d = v.dmax[e];
    if (d > m) m = d;
  }
  red[threadIdx.x] = m;
  __syncthreads();
  for (int h = 128; h > 0; h >>= 1) {
    if ((int)threadIdx.x < h && red[threadIdx.x + h] > red[threadIdx.x]) red[threadIdx.x] = red[threadIdx.x + h];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[sub] = red[0];
}
// the sums of the single engine (the same slices, CTA per slice), then per submodel the slices
// added in order into out[8 sub + slot]
enum SumWhat { SUM_RINT, SUM_BB, SUM_RZ, SUM_PQ, SUM_RR, SUM_UPD };
__global__ void __launch_bounds__(SUMS_THREADS) kb_sums_slice(Seg g, const SubView* __restrict__ V, int what) {
  __shared__ double s0[SUMS_THREADS], s1[SUMS_THREADS];
  const int sq = seg_find(g, blockIdx.x), sub = g.sub[sq];
  const SubView& v = V[sub];
  const int c = blockIdx.x - g.start[sq];
  switch (what) {
    case SUM_RINT: sub_sums_slice(v.ndof, c, 0, v.rint, nullptr, v.isC, v.sumPart, s0, s1); break;
    case SUM_BB: sub_sums_slice(v.ndof, c, 1, v.b, v.b, v.isC, v.sumPart, s0, s1); break;
    case SUM_RZ: sub_sums_slice(v.ndof, c, 1, v.r, v.z, v.isC, v.sumPart, s0, s1); break;
    case SUM_PQ: sub_sums_slice(v.ndof, c, 1, v.p, v.q, v.isC, v.sumPart, s0, s1); break;
    case SUM_RR: sub_sums_slice(v.ndof, c, 1, v.r, v.r, v.isC, v.sumPart, s0, s1); break;
    default: sub_sums_slice(v.ndof, c, 2, v.x, v.u, v.isC, v.sumPart, s0, s1); break;
  }
}
__global__ void kb_sums_final(Seg g, const SubView* __restrict__ V, double* __restrict__ out, int slot) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= g.n) return;
  const int sub = g.sub[q];
  sub_sums_final(V[sub].ndof, V[sub].sumPart, out + 8 * sub + slot);
}
__global__ void kb_scale_s(Seg g, const SubView* __restrict__ V) {
  SB_ITEM(blockDim.x);
  if (item < v.nn) sub_scale_s_node(item, v.diag, v.val, v.s);
}
__global__ void kb_scale_vals(Seg g, const SubView* __restrict__ V) {
  SB_ITEM(blockDim.x);
  if (item < v.nbk) sub_scale_vals_block(item, v.blkRow, v.col, v.s, v.val, v.vals);
}
__global__ void kb_rhs(Seg g, const SubView* __restrict__ V) {
  SB_ITEM(blockDim.x);
  if (item < v.ndof) sub_rhs_dof(item, v.rint, v.isC, v.s, v.b, v.r, v.x);
}
__global__ void kb_spmv(Seg g, const SubView* __restrict__ V) {
  SB_ITEM(blockDim.x);
  if (item < v.nn) sub_spmv_node(item, v.rowPtr, v.col, v.vals, v.p, v.q);
}
// alpha = rz / pq from the submodel's scalars S[a] and S[4]
__global__ void kb_axpy2(Seg g, const SubView* __restrict__ V, const double* __restrict__ S, int a) {
  SB_ITEM(blockDim.x);
  if (item < v.ndof) sub_axpy2_dof(item, S[8 * sub + a], S[8 * sub + 4], v.p, v.q, v.x, v.r);
}
// beta = S[2 - a] / S[a]
__global__ void kb_xpby(Seg g, const SubView* __restrict__ V, const double* __restrict__ S, int a) {
  SB_ITEM(blockDim.x);
  if (item < v.ndof) sub_xpby_dof(item, S[8 * sub + 2 - a], S[8 * sub + a], v.z, v.p);
}
__global__ void kb_copy_zp(Seg g, const SubView* __restrict__ V) {
  SB_ITEM(blockDim.x);
  if (item < v.ndof) v.p[item] = v.z[item];
}
__global__ void kb_mul(Seg g, const SubView* __restrict__ V) {
  SB_ITEM(blockDim.x);
  if (item < v.ndof) v.x[item] *= v.s[item];
}
__global__ void kb_line_factor(Seg g, const SubView* __restrict__ V) {
  SB_ITEM(blockDim.x);
  if (item < v.ncol) sub_line_factor_column(item, v.nz, v.diag, v.subBlk, v.vals, v.lf);
}
__global__ void kb_line_apply(Seg g, const SubView* __restrict__ V) {
  SB_ITEM(blockDim.x);
  if (item < v.ncol) sub_line_apply_column(item, v.nz, v.lf, v.r, v.z);
}
__global__ void kb_commit_points(Seg g, const SubView* __restrict__ V) {
  SB_ITEM(blockDim.x);
  if (item < v.npts) commit(v.pts[item]);
}
__global__ void __launch_bounds__(32 * SA_WARPS) kb_commit_elastic(Seg g, const SubView* __restrict__ V) {
  __shared__ CommitSmem sm[SA_WARPS];
  const int sq = seg_find(g, blockIdx.x), sub = g.sub[sq];
  const SubView& v = V[sub];
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int e = (blockIdx.x - g.start[sq]) * SA_WARPS + w;
  if (e >= v.ne || v.eAn[e] >= 0) return;
  sub_commit_elastic_element(e, lane, sm[w], v.conn, v.eMat, v.eBb, v.Bm, v.Bw, v.u, v.uN, v.elas, v.sigE, v.eFn);
}
__global__ void kb_copy_uN(Seg g, const SubView* __restrict__ V) {
  SB_ITEM(blockDim.x);
  if (item < v.ndof) v.uN[item] = v.u[item];
}
#undef SB_ITEM

// per submodel: where it is in run()'s history loop and in its current stepTo
enum RunPhase { RP_START, RP_NEWTON, RP_DONE, RP_FAILED };
struct RunState {
  RunPhase ph = RP_START;
  int k = 1, nsub = 1, nsubNext = 1, attempt = 0, sIdx = 1, sample = 0;
  double snapTn = 0, dLast = 0;
  long long totalNewton = 0;
  int cutbacks = 0, steps = 0;
  std::vector<double> Wdie, Wsub, Edie, Esub;
  double T = 0, dt = 0, rPrev = INFINITY, dMax = 0, tol = 0, bn = 0;
  int it = 1;
  bool haveK = false, wantK = false;
  tm_status status = TM_OK;
};

struct Batch {
  std::vector<SubModel*> M;
  int B = 0;
  cudaStream_t st = nullptr;
  std::vector<cudaStream_t> own;         // the submodels' own streams, restored at the end
  DBuf<SubView> dV;
  DBuf<SubRound> dR;
  DBuf<double> dS, dN, dDmax, dElas;     // PCG scalars (8 per submodel), norms (8 per), plastic increments, records
  std::vector<SubRound> R;
  std::vector<double> hS, hN, hDmax, hElas;
  int recMax = 0;

  explicit Batch(const std::vector<SubModel*>& subs) : M(subs), B((int)subs.size()) {
    TM_CUDA_CHECK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    for (SubModel* m : M) {
      TM_CUDA_CHECK(cudaStreamSynchronize(m->st));
      own.push_back(m->st);
      m->st = st;                         // the submodel's own operations join the batch's stream
      recMax = std::max(recMax, m->nrec);
    }
    hElas.assign((size_t)B * recMax * 42, 0.0);
    dElas.alloc(hElas.size());
    std::vector<SubView> hv(B);
    for (int s = 0; s < B; s++) {
      SubModel& m = *M[s];
      SubView& v = hv[s];
      v.ne = m.ne; v.nn = m.nn; v.ndof = m.ndof; v.nbk = m.nbk; v.nbnd = m.nbnd; v.ncol = m.nx * m.ny; v.nz = m.nz;
      v.npts = 8 * m.nsolderE;
      v.conn = m.d_conn.p; v.eMat = m.d_eMat.p; v.eBb = m.d_eBb.p; v.eAn = m.d_eAn.p; v.rowPtr = m.d_rowPtr.p; v.col = m.d_col.p;
      v.diag = m.d_diag.p; v.blkRow = m.d_blkRow.p; v.blkStart = m.d_blkStart.p; v.blkList = m.d_blkList.p;
      v.nodeStart = m.d_nodeStart.p; v.nodeList = m.d_nodeList.p; v.bNodes = m.d_bNodes.p; v.bGlob = m.d_bGlob.p; v.subBlk = m.d_subBlk.p;
      v.isC = m.d_isC.p; v.Bm = m.d_Bm.p; v.Bw = m.d_Bw.p; v.bW = m.d_bW.p; v.u25 = m.d_u25.p;
      v.elas = dElas.p + (size_t)s * recMax * 42;
      v.u = m.d_u.p; v.uN = m.d_uN.p; v.sigE = m.d_sigE.p; v.eFn = m.d_eFn.p; v.eK = m.d_eK.p; v.eF = m.d_eF.p; v.fe = m.d_fe.p;
      v.dmax = m.d_dmax.p; v.val = m.d_val.p; v.vals = m.d_vals.p; v.s = m.d_s.p; v.rint = m.d_rint.p; v.b = m.d_b.p; v.r = m.d_r.p;
      v.z = m.d_z.p; v.p = m.d_p.p; v.q = m.d_q.p; v.x = m.d_x.p; v.lf = m.d_lf.p; v.sumPart = m.d_sumPart.p; v.pts = m.d_pts.p;
      // the batch owns the material records: the single engine uploads its own again when next used
      m.haveKey = false;
    }
    dV.upload(hv, st);
    R.assign(B, SubRound{});
    dR.alloc(B);
    hS.assign(8 * (size_t)B, 0.0); dS.alloc(hS.size());
    hN.assign(8 * (size_t)B, 0.0); dN.alloc(hN.size());
    hDmax.assign(B, 0.0); dDmax.alloc(B);
  }
  ~Batch() {
    cudaStreamSynchronize(st);
    for (int s = 0; s < B; s++) { M[s]->st = own[s]; M[s]->haveKey = false; }
    cudaStreamDestroy(st);
  }

  // a segment over the listed submodels, count(s) items each, per items per CTA; false when empty
  template <class F>
  static bool seg(Seg& g, const std::vector<int>& subs, F count, int per) {
    g.n = 0;
    long long tot = 0;
    for (int s : subs) {
      const long long c = count(s);
      if (c <= 0) continue;
      g.sub[g.n] = s;
      g.start[g.n] = (int)tot;
      tot += (c + per - 1) / per;
      g.n++;
    }
    if (tot >= (1LL << 31)) fail(TM_BAD_INPUT, "submodel batch too large for one launch");
    g.start[g.n] = (int)tot;
    return tot > 0;
  }
  static Seg one_each(const std::vector<int>& subs) {
    Seg g;
    g.n = (int)subs.size();
    for (int q = 0; q < g.n; q++) { g.sub[q] = subs[q]; g.start[q] = q; }
    g.start[g.n] = g.n;
    return g;
  }
  void upload_rounds() { TM_CUDA_CHECK(cudaMemcpyAsync(dR.p, R.data(), B * sizeof(SubRound), cudaMemcpyHostToDevice, st)); }

  void prescribe(const std::vector<int>& subs) {
    Seg g;
    if (!seg(g, subs, [&](int s) { return M[s]->nbnd; }, 128)) return;
    upload_rounds();
    note_launch();
    kb_prescribe<<<g.start[g.n], 128, 0, st>>>(g, dV.p, dR.p);
    TM_CUDA_CHECK(cudaGetLastError());
  }

  // assemble (13-fatigue.js:776-853) of the listed submodels with their R[s]; the plastic
  // increments go to dDmax
  void assemble(const std::vector<int>& subs, bool anyFresh) {
    upload_rounds();
    if (anyFresh) TM_CUDA_CHECK(cudaMemcpyAsync(dElas.p, hElas.data(), hElas.size() * sizeof(double), cudaMemcpyHostToDevice, st));
    Seg g;
    note_launch(3);
    if (seg(g, subs, [&](int s) { return M[s]->ne; }, SA_WARPS)) kb_assemble<<<g.start[g.n], 32 * SA_WARPS, 0, st>>>(g, dV.p, dR.p);
    if (seg(g, subs, [&](int s) { return M[s]->ndof; }, 256)) kb_gather_rint<<<g.start[g.n], 256, 0, st>>>(g, dV.p);
    std::vector<int> wk;
    for (int s : subs) if (R[s].wantK) wk.push_back(s);
    if (seg(g, wk, [&](int s) { return M[s]->nbk; }, 128)) { note_launch(); kb_gather_val<<<g.start[g.n], 128, 0, st>>>(g, dV.p); }
    kb_dmax<<<(int)subs.size(), 256, 0, st>>>(one_each(subs), dV.p, dDmax.p);
    TM_CUDA_CHECK(cudaGetLastError());
  }

  void sums(const std::vector<int>& subs, int what, DBuf<double>& out, int slot) {
    Seg g;
    if (!seg(g, subs, [&](int s) { return sums_parts(M[s]->ndof); }, 1)) return;
    note_launch(2);
    kb_sums_slice<<<g.start[g.n], SUMS_THREADS, 0, st>>>(g, dV.p, what);
    kb_sums_final<<<1, SB_MAX, 0, st>>>(one_each(subs), dV.p, out.p, slot);
    TM_CUDA_CHECK(cudaGetLastError());
  }
  void fetch(DBuf<double>& d, std::vector<double>& h) {
    TM_CUDA_CHECK(cudaMemcpyAsync(h.data(), d.p, h.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
    TM_CUDA_CHECK(cudaStreamSynchronize(st));
  }
  template <class K>
  void each_dof(const std::vector<int>& subs, K kern) {
    Seg g;
    if (seg(g, subs, [&](int s) { return M[s]->ndof; }, 256)) { note_launch(); kern<<<g.start[g.n], 256, 0, st>>>(g, dV.p); }
  }

  // z = M^-1 r: the z-line submodels in one launch, the IC(0) ones through their level launches
  void pc_apply(const std::vector<int>& subs) {
    std::vector<int> line;
    for (int s : subs) {
      if (M[s]->precond == TM_SUB_PC_LINE) line.push_back(s);
      else M[s]->pc_apply(M[s]->d_r.p, M[s]->d_z.p);
    }
    Seg g;
    if (seg(g, line, [&](int s) { return (long long)M[s]->nx * M[s]->ny; }, 128)) {
      note_launch();
      kb_line_apply<<<g.start[g.n], 128, 0, st>>>(g, dV.p);
    }
    TM_CUDA_CHECK(cudaGetLastError());
  }

  // _solve (13-fatigue.js:886-917) for the listed submodels, each to its RunState tol: d_x = the
  // Newton increment
  void solve(const std::vector<int>& subs, std::vector<RunState>& rs) {
    Seg g;
    note_launch(3);
    if (seg(g, subs, [&](int s) { return M[s]->nn; }, 128)) kb_scale_s<<<g.start[g.n], 128, 0, st>>>(g, dV.p);
    if (seg(g, subs, [&](int s) { return M[s]->nbk; }, 128)) kb_scale_vals<<<g.start[g.n], 128, 0, st>>>(g, dV.p);
    each_dof(subs, kb_rhs);
    std::vector<int> line;
    for (int s : subs) {
      SubModel& m = *M[s];
      if (m.precond == TM_SUB_PC_LINE) line.push_back(s);
      else if (!m.pcBuilt || m.pcStale) { ic_factor(m.ic, m.d_vals.p, st); m.pcBuilt = true; m.pcStale = false; m.pcIters = 0; }
    }
    if (seg(g, line, [&](int s) { return (long long)M[s]->nx * M[s]->ny; }, 128)) {
      note_launch();
      kb_line_factor<<<g.start[g.n], 128, 0, st>>>(g, dV.p);
    }
    sums(subs, SUM_BB, dN, 0);
    fetch(dN, hN);
    std::vector<int> act;
    for (int s : subs) {
      rs[s].bn = std::sqrt(hN[8 * s]);
      if (rs[s].bn != 0) act.push_back(s);
    }
    if (act.empty()) return;
    const std::vector<int> solved = act;
    pc_apply(act);
    each_dof(act, kb_copy_zp);
    int a = 0;
    sums(act, SUM_RZ, dS, a);
    std::vector<int> its(B, 0);
    int it;
    for (it = 1; it <= 2000 && !act.empty(); it++) {
      Seg ga;
      if (seg(ga, act, [&](int s) { return M[s]->nn; }, 128)) { note_launch(); kb_spmv<<<ga.start[ga.n], 128, 0, st>>>(ga, dV.p); }
      sums(act, SUM_PQ, dS, 4);
      if (seg(ga, act, [&](int s) { return M[s]->ndof; }, 256)) { note_launch(); kb_axpy2<<<ga.start[ga.n], 256, 0, st>>>(ga, dV.p, dS.p, a); }
      sums(act, SUM_RR, dS, 6);
      fetch(dS, hS);
      std::vector<int> next;
      for (int s : act) {
        if (std::sqrt(hS[8 * s + 6]) / rs[s].bn < rs[s].tol) its[s] = it;
        else next.push_back(s);
      }
      act.swap(next);
      if (act.empty()) break;
      pc_apply(act);
      sums(act, SUM_RZ, dS, 2 - a);
      if (seg(ga, act, [&](int s) { return M[s]->ndof; }, 256)) { note_launch(); kb_xpby<<<ga.start[ga.n], 256, 0, st>>>(ga, dV.p, dS.p, a); }
      a = 2 - a;
    }
    for (int s : act) its[s] = 2001;   // the loop's bound, as the single engine's counter ends
    each_dof(solved, kb_mul);
    TM_CUDA_CHECK(cudaGetLastError());
    for (int s : solved) {
      SubModel& m = *M[s];
      m.pcgSolves++;
      m.pcgIters += its[s];
      if (m.precond == TM_SUB_PC_LINE) continue;
      if (!m.pcIters) m.pcIters = its[s];
      else if (its[s] > 2 * m.pcIters) m.pcStale = true;
    }
  }

  // the end of a converged stepTo: the solder points' trial states become committed, the elastic
  // elements' stresses and forces are updated and u_n = u
  void commit(const std::vector<int>& subs) {
    Seg g;
    if (seg(g, subs, [&](int s) { return 8LL * M[s]->nsolderE; }, 128)) { note_launch(); kb_commit_points<<<g.start[g.n], 128, 0, st>>>(g, dV.p); }
    if (seg(g, subs, [&](int s) { return M[s]->ne; }, SA_WARPS)) {
      note_launch();
      kb_commit_elastic<<<g.start[g.n], 32 * SA_WARPS, 0, st>>>(g, dV.p);
    }
    each_dof(subs, kb_copy_uN);
    TM_CUDA_CHECK(cudaGetLastError());
  }
};

}  // namespace

void submodel_run_batch(const std::vector<SubModel*>& subs, int nsteps, const double* ht, const double* hT, const int* hcycle, int cycles,
                        const double* cphi, const double* sphi, double* out10, double* perCycle, double* loop, int32_t* status) {
  const int n = (int)subs.size();
  if (nsteps < 2 || cycles < 1) fail(TM_BAD_INPUT, "submodel run: need >= 2 history points and >= 1 cycle");
  for (int k = 0; k < nsteps; k++) if (hcycle[k] < 0 || hcycle[k] > cycles) fail(TM_BAD_INPUT, "submodel run: cycle index out of range");
  for (int b0 = 0; b0 < n; b0 += SB_MAX) {
    const int nb = std::min(SB_MAX, n - b0);
    std::vector<SubModel*> part(subs.begin() + b0, subs.begin() + b0 + nb);
    Batch bt(part);
    std::vector<RunState> rs(nb);
    auto begin_substep = [&](int s) {
      RunState& r = rs[s];
      const double T0 = hT[r.k - 1], T1 = hT[r.k], t0s = ht[r.k - 1], t1s = ht[r.k];
      r.T = T0 + (T1 - T0) * r.sIdx / r.nsub;
      r.dt = (t1s - t0s) / r.nsub;
      r.ph = RP_START;
    };
    auto begin_attempt = [&](int s) {
      rs[s].snapTn = part[s]->Tn;
      part[s]->snapshot();
      rs[s].sIdx = 1;
      begin_substep(s);
    };
    auto finish = [&](int s) {
      RunState& r = rs[s];
      const int nc = cycles;
      const double dWdie = r.Wdie[nc] - r.Wdie[nc - 1], dWsub = r.Wsub[nc] - r.Wsub[nc - 1];
      const double dEdie = r.Edie[nc] - r.Edie[nc - 1], dEsub = r.Esub[nc] - r.Esub[nc - 1];
      const double dW = std::max(dWdie, dWsub), dE = dWdie >= dWsub ? dEdie : dEsub;
      const double prev = nc >= 2 ? std::max(r.Wdie[nc - 1] - r.Wdie[nc - 2], r.Wsub[nc - 1] - r.Wsub[nc - 2]) : NAN;
      const double stab = std::isfinite(prev) && prev > 0 ? std::fabs(dW - prev) / prev : NAN;
      const double o[10] = {dW, dWdie, dWsub, dE, dEdie, dEsub, stab, (double)r.steps, (double)r.cutbacks,
                            (double)r.totalNewton / std::max(r.steps, 1)};
      std::copy(o, o + 10, out10 + 10 * (size_t)(b0 + s));
      double* pc = perCycle + 2 * (size_t)cycles * (b0 + s);
      for (int c = 1; c <= nc; c++) { pc[2 * (c - 1)] = r.Wdie[c] - r.Wdie[c - 1]; pc[2 * (c - 1) + 1] = r.Wsub[c] - r.Wsub[c - 1]; }
      r.ph = RP_DONE;
    };
    auto attempt_failed = [&](int s) {
      RunState& r = rs[s];
      part[s]->restore(r.snapTn);
      r.nsub *= 2;
      r.cutbacks++;
      if (++r.attempt >= 8) { r.status = TM_NOT_CONVERGED; r.ph = RP_FAILED; return; }
      begin_attempt(s);
    };
    auto substep_done = [&](int s) {
      RunState& r = rs[s];
      if (++r.sIdx <= r.nsub) { begin_substep(s); return; }
      // the history step is complete
      r.nsubNext = r.dLast > 0.5 * INELASTIC_STEP_MAX ? std::min(r.nsub * 2, 64)
                                                        : (r.dLast < 0.2 * INELASTIC_STEP_MAX ? std::max(1, r.nsub >> 1) : r.nsub);
      double avg[4];
      part[s]->sample_loop(hT[r.k], cphi[b0 + s], sphi[b0 + s], loop + 4 * (size_t)nsteps * (b0 + s) + 4 * (size_t)r.sample++);
      part[s]->layer_avg(avg);
      const int c = hcycle[r.k];
      r.Wdie[c] = avg[0]; r.Edie[c] = avg[1]; r.Wsub[c] = avg[2]; r.Esub[c] = avg[3];
      if (++r.k >= nsteps) { finish(s); return; }
      r.nsub = r.nsubNext;
      r.attempt = 0;
      begin_attempt(s);
    };
    for (int s = 0; s < nb; s++) {
      RunState& r = rs[s];
      if (!part[s]->nsolderE || part[s]->elasticSolder) { r.status = TM_BAD_INPUT; r.ph = RP_FAILED; continue; }
      r.Wdie.assign(cycles + 1, 0.0); r.Wsub = r.Wdie; r.Edie = r.Wdie; r.Esub = r.Wdie;
      part[s]->sample_loop(25, cphi[b0 + s], sphi[b0 + s], loop + 4 * (size_t)nsteps * (b0 + s) + 4 * (size_t)r.sample++);
      begin_attempt(s);
    }
    for (;;) {
      // stepTo's start: prescribe the cut boundary
      std::vector<int> start, newton;
      for (int s = 0; s < nb; s++)
        if (rs[s].ph == RP_START) {
          RunState& r = rs[s];
          part[s]->prescribe_args(r.T, &bt.R[s].fa, &bt.R[s].fb, &bt.R[s].t);
          r.ph = RP_NEWTON; r.it = 1; r.rPrev = INFINITY; r.haveK = false;
          start.push_back(s);
        }
      bt.prescribe(start);
      for (int s = 0; s < nb; s++) if (rs[s].ph == RP_NEWTON) newton.push_back(s);
      if (newton.empty()) break;
      // one Newton iteration of every submodel in a stepTo
      bool anyFresh = false;
      for (int s : newton) {
        RunState& r = rs[s];
        SubModel& m = *part[s];
        r.wantK = r.it <= 2 || !r.haveK;
        SubRound& R = bt.R[s];
        R.fresh = m.fresh_for(r.T);
        if (R.fresh) { m.fill_records(r.T, bt.hElas.data() + (size_t)s * bt.recMax * 42); anyFresh = true; }
        m.step_params(r.T, r.dt, &R.kc, &R.fSolder);
        R.P = m.P;
        R.wantK = r.wantK;
      }
      bt.assemble(newton, anyFresh);
      for (int s : newton) {
        RunState& r = rs[s];
        SubModel& m = *part[s];
        if (r.wantK) r.haveK = true;
        m.haveKey = true; m.keyTn = m.Tn; m.keyT = r.T;
      }
      bt.sums(newton, SUM_RINT, bt.dN, 0);
      bt.fetch(bt.dN, bt.hN);
      bt.fetch(bt.dDmax, bt.hDmax);
      std::vector<int> conv, solve, refresh;
      for (int s : newton) {
        RunState& r = rs[s];
        r.dMax = bt.hDmax[s];
        const double rn = std::sqrt(bt.hN[8 * s]), fn = std::sqrt(bt.hN[8 * s + 1]);
        const double ref = std::max(fn, 1e-30);
        if (rn / ref < SUB_RES_TOL) { conv.push_back(s); continue; }
        if (!r.wantK && rn > 0.5 * r.rPrev) refresh.push_back(s);   // stalled with the frozen tangent: refresh it
        r.rPrev = rn;
        r.tol = std::max(SUB_INNER_TOL, std::min(1e-3, 0.01 * SUB_RES_TOL * ref / std::max(rn, 1e-300)));
        solve.push_back(s);
      }
      if (!refresh.empty()) {
        for (int s : refresh) { bt.R[s].fresh = 0; bt.R[s].wantK = 1; }
        bt.assemble(refresh, false);
      }
      if (!solve.empty()) {
        bt.solve(solve, rs);
        bt.sums(solve, SUM_UPD, bt.dN, 0);   // u += du on the free DOFs
        bt.fetch(bt.dN, bt.hN);
        for (int s : solve) {
          RunState& r = rs[s];
          const bool done = std::sqrt(bt.hN[8 * s]) < SUB_DU_TOL * std::max(std::sqrt(bt.hN[8 * s + 1]), 1e-30);
          r.it++;
          if (done) conv.push_back(s);
          else if (r.it > SUB_NEWTON_MAXIT) {   // not converged: the attempt fails
            r.totalNewton += r.it; r.steps++; r.dLast = r.dMax;
            attempt_failed(s);
          }
        }
      }
      if (conv.empty()) continue;
      // converged stepTo: the final assembly and the commit
      for (int s : conv) { bt.R[s].fresh = 0; bt.R[s].wantK = 0; }
      bt.assemble(conv, false);
      bt.commit(conv);
      bt.fetch(bt.dDmax, bt.hDmax);
      for (int s : conv) {
        RunState& r = rs[s];
        part[s]->Tn = r.T;
        r.totalNewton += r.it; r.steps++;
        r.dLast = bt.hDmax[s];
        if (r.dLast > INELASTIC_STEP_MAX) attempt_failed(s);
        else substep_done(s);
      }
    }
    for (int s = 0; s < nb; s++) status[b0 + s] = rs[s].status;
  }
}

}  // namespace tmg
