// Per-step numeric set-up on the GPU: element condensation, stencil assembly, constraints,
// Jacobi scaling, level-0 column factors, transfer weights and shell column factors (the
// Galerkin products and the coarsest factor are in tm_coarse.cu).
//
// This file is compiled with -fmad=false: every quantity here is then computed with the same
// operations in the same order as the reference (JavaScript has no fused multiply-add), so the
// assembled operator is bit-identical to the FP64 oracle.
//
// Reference lines followed:
//   shapeMatrices / elementK33Fast / elementFth   src/core/09-assembly.js:69-133 (UNIV :26-60)
//   condense33 (cholDense 1e-14)                  src/core/07-element.js:88-121, 01-util.js:70-107
//   assembleStep (element order summation)        src/core/09-assembly.js:392-424
//   applyConstraints                              src/core/09-assembly.js:445-464
//   LinearSolver._scale                           src/core/10-solver.js:852-866
//   factorColumns / chol3                         src/core/10-solver.js:12-68
//   shellWeights                                  src/core/10-solver.js:337-353
//   factorShellColumns                            src/core/10-solver.js:474-494
#include <cmath>
#include <cstring>

#include <math_constants.h>

#include "tm_internal.h"

namespace tmg {

namespace {

const int HEX_XI[8] = {-1, 1, 1, -1, -1, 1, 1, -1};
const int HEX_ETA[8] = {-1, -1, 1, 1, -1, -1, 1, 1};
const int HEX_ZETA[8] = {-1, -1, -1, -1, 1, 1, 1, 1};
const int VOIGT[3][3] = {{0, 3, 5}, {3, 1, 4}, {5, 4, 2}};

struct Univ {
  double G[3 * 9 * 121], g[3 * 3 * 11], GH[9 * 121], gH[3 * 11];
};

// UNIV (09-assembly.js:26-60): natural-coordinate integrals of the 11 functions
const Univ& univ() {
  static Univ U;
  static bool done = false;
  if (done) return U;
  std::memset(&U, 0, sizeof(U));
  const double GP2 = 1 / std::sqrt(3.0);
  const double simpson[3] = {1.0 / 3, 4.0 / 3, 1.0 / 3};
  double d[3][11];
  for (int j = 0; j < 3; j++) {
    const double zeta = j - 1;
    for (int ip = 0; ip < 4; ip++) {
      const double xi = (ip & 1) ? GP2 : -GP2, eta = (ip & 2) ? GP2 : -GP2;
      for (int a = 0; a < 8; a++) {
        const double xa = HEX_XI[a], ya = HEX_ETA[a], za = HEX_ZETA[a];
        d[0][a] = xa * (1 + ya * eta) * (1 + za * zeta) * 0.125;
        d[1][a] = ya * (1 + xa * xi) * (1 + za * zeta) * 0.125;
        d[2][a] = za * (1 + xa * xi) * (1 + ya * eta) * 0.125;
      }
      d[0][8] = -2 * xi; d[1][8] = 0; d[2][8] = 0;
      d[0][9] = 0; d[1][9] = -2 * eta; d[2][9] = 0;
      d[0][10] = 0; d[1][10] = 0; d[2][10] = -2 * zeta;
      for (int r = 0; r < 3; r++)
        for (int a = 0; a < 11; a++) {
          U.g[(j * 3 + r) * 11 + a] += d[r][a];
          U.gH[r * 11 + a] += simpson[j] * d[r][a];
          for (int s = 0; s < 3; s++)
            for (int b = 0; b < 11; b++) {
              const double v = d[r][a] * d[s][b];
              U.G[((j * 9 + r * 3 + s) * 121) + a * 11 + b] += v;
              U.GH[(r * 3 + s) * 121 + a * 11 + b] += simpson[j] * v;
            }
        }
    }
  }
  done = true;
  return U;
}

// shapeMatrices (09-assembly.js:69-93): M (6 x 33 x 33) from D (36) or the layered weights W (108)
void shape_matrices(const double* Wst, const double* D, double* M) {
  const Univ& U = univ();
  std::fill(M, M + 6 * 1089, 0.0);
  const int nst = D ? 1 : 3;
  const int PAIR[6][3] = {{0, 0, 0}, {1, 1, 1}, {2, 2, 2}, {3, 0, 1}, {4, 1, 2}, {5, 2, 0}};
  for (int j = 0; j < nst; j++) {
    const double* Wj = D ? D : Wst + 36 * j;
    for (int pi = 0; pi < 6; pi++) {
      const int m = PAIR[pi][0], r = PAIR[pi][1], s = PAIR[pi][2];
      double* Mm = M + m * 1089;
      const int rs[2][2] = {{r, s}, {s, r}};
      const int nrs = r == s ? 1 : 2;
      for (int t = 0; t < nrs; t++) {
        const int rr = rs[t][0], ss = rs[t][1];
        const double* Gb = D ? U.GH + (rr * 3 + ss) * 121 : U.G + (j * 9 + rr * 3 + ss) * 121;
        for (int p = 0; p < 3; p++)
          for (int q = 0; q < 3; q++) {
            const double dv = Wj[VOIGT[p][rr] * 6 + VOIGT[q][ss]];
            if (dv == 0) continue;
            for (int a = 0; a < 11; a++) {
              const int row = (3 * a + p) * 33 + q, ga = a * 11;
              for (int b = 0; b < 11; b++) Mm[row + 3 * b] += dv * Gb[ga + b];
            }
          }
      }
    }
  }
}

// elementFth (09-assembly.js:115-133)
void element_fth(double hx, double hy, double hz, const double* Sst, const double* s0, double* f) {
  const Univ& U = univ();
  std::fill(f, f + 33, 0.0);
  const double h[3] = {hx, hy, hz};
  const double V8 = hx * hy * hz / 8;
  const int nst = s0 ? 1 : 3;
  for (int j = 0; j < nst; j++) {
    const double* Sj = s0 ? s0 : Sst + 6 * j;
    for (int r = 0; r < 3; r++) {
      const double c = V8 * (2 / h[r]);
      const double* gb = s0 ? U.gH + r * 11 : U.g + (j * 3 + r) * 11;
      for (int p = 0; p < 3; p++) {
        const double sv = c * Sj[VOIGT[p][r]];
        if (sv == 0) continue;
        for (int a = 0; a < 11; a++) f[3 * a + p] += sv * gb[a];
      }
    }
  }
}

inline int grid_for(size_t n, int block) { return (int)((n + block - 1) / block); }

// ---- device helpers --------------------------------------------------------------------------
// cholDense (01-util.js:70-91) on a 9x9 matrix, one thread
__device__ void chol_dense9(double* A, double rel) {
  double dmax = 0;
  for (int i = 0; i < 9; i++) dmax = fmax(dmax, fabs(A[i * 9 + i]));
  const double jitter = rel * (dmax != 0 ? dmax : 1);
  for (int j = 0; j < 9; j++) {
    const int rj = j * 9;
    double d = A[rj + j];
    for (int k = 0; k < j; k++) d -= A[rj + k] * A[rj + k];
    if (!(d > jitter)) d = fmax(fabs(d), jitter);
    const double ljj = sqrt(d);
    A[rj + j] = ljj;
    const double inv = 1 / ljj;
    for (int i = j + 1; i < 9; i++) {
      const int ri = i * 9;
      double s = A[ri + j];
      for (int k = 0; k < j; k++) s -= A[ri + k] * A[rj + k];
      A[ri + j] = s * inv;
    }
  }
}

// cholSolveDense (01-util.js:94-107)
__device__ void chol_solve9(const double* L, double* b) {
  for (int i = 0; i < 9; i++) {
    double s = b[i];
    for (int k = 0; k < i; k++) s -= L[i * 9 + k] * b[k];
    b[i] = s / L[i * 9 + i];
  }
  for (int i = 8; i >= 0; i--) {
    double s = b[i];
    for (int k = i + 1; k < 9; k++) s -= L[k * 9 + i] * b[k];
    b[i] = s / L[i * 9 + i];
  }
}

// ---- element classes: K33 = sum_m c_m M^m, condensation (one warp per class) ------------------
__global__ void k_class_condense(int ncls, const int* __restrict__ clsPset, const double* __restrict__ clsH,
                                 const double* __restrict__ psetM, const double* __restrict__ clsF33,
                                 const int* __restrict__ clsBorn, double* __restrict__ clsKc, double* __restrict__ clsFc) {
  extern __shared__ double sm[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int cls = blockIdx.x * (blockDim.x >> 5) + warp;
  if (cls >= ncls) return;
  double* K = sm + warp * 2048;        // 1089
  double* Kc = K + 1089;               // 576
  double* X = Kc + 576;                // 216
  double* Kaa = X + 216;               // 81
  double* xf = Kaa + 81;               // 9 (+ pad)
  const double hx = clsH[3 * cls], hy = clsH[3 * cls + 1], hz = clsH[3 * cls + 2];
  const double V8 = hx * hy * hz / 8;
  const double c0 = V8 * 4 / (hx * hx), c1 = V8 * 4 / (hy * hy), c2 = V8 * 4 / (hz * hz);
  const double c3 = V8 * 4 / (hx * hy), c4 = V8 * 4 / (hy * hz), c5 = V8 * 4 / (hz * hx);
  const double* M = psetM + (size_t)clsPset[cls] * 6 * 1089;
  // elementK33Fast (09-assembly.js:96-108): upper triangle, then mirrored
  for (int o = lane; o < 1089; o += 32) {
    const int i = o / 33, j = o % 33;
    if (j >= i) K[o] = c0 * M[o] + c1 * M[1089 + o] + c2 * M[2178 + o] + c3 * M[3267 + o] + c4 * M[4356 + o] + c5 * M[5445 + o];
  }
  __syncwarp();
  for (int o = lane; o < 1089; o += 32) {
    const int i = o / 33, j = o % 33;
    if (j < i) K[o] = K[j * 33 + i];
  }
  __syncwarp();
  if (lane == 0) {
    for (int i = 0; i < 9; i++)
      for (int j = 0; j < 9; j++) Kaa[i * 9 + j] = K[(24 + i) * 33 + 24 + j];
    chol_dense9(Kaa, 1e-14);
  }
  __syncwarp();
  if (lane < 24) {
    double col[9];
    for (int i = 0; i < 9; i++) col[i] = K[(24 + i) * 33 + lane];
    chol_solve9(Kaa, col);
    for (int i = 0; i < 9; i++) X[i * 24 + lane] = col[i];
  }
  __syncwarp();
  for (int e = lane; e < 576; e += 32) {
    const int i = e / 24, j = e % 24;
    double s = K[i * 33 + j];
    for (int q = 0; q < 9; q++) s -= K[i * 33 + 24 + q] * X[q * 24 + j];
    Kc[e] = s;
  }
  __syncwarp();
  // exact symmetry (07-element.js:108)
  for (int e = lane; e < 576; e += 32) {
    const int i = e / 24, j = e % 24;
    if (j > i) {
      const double v = 0.5 * (Kc[i * 24 + j] + Kc[j * 24 + i]);
      Kc[i * 24 + j] = v;
      Kc[j * 24 + i] = v;
    }
  }
  __syncwarp();
  double* outK = clsKc + (size_t)cls * 576;
  for (int e = lane; e < 576; e += 32) outK[e] = Kc[e];
  if (clsBorn[cls]) {
    const double* f = clsF33 + (size_t)cls * 33;
    if (lane == 0) {
      for (int i = 0; i < 9; i++) xf[i] = f[24 + i];
      chol_solve9(Kaa, xf);
    }
    __syncwarp();
    if (lane < 24) {
      double s = f[lane];
      for (int q = 0; q < 9; q++) s -= K[lane * 33 + 24 + q] * xf[q];
      clsFc[(size_t)cls * 24 + lane] = s;
    }
  } else if (lane < 24) {
    clsFc[(size_t)cls * 24 + lane] = 0;
  }
}

// directional derivative of the condensation, one warp per class: with K the class's K33, dK its
// derivative along the direction (the same shape-matrix sum over the direction's data), and
// X = Kaa^-1 Kau, y = Kaa^-1 fa: dKc = dKuu - dKua X - X^T dKau + X^T dKaa X and
// dfc = dfu - dKua y - X^T dfa + X^T dKaa y, then the exact symmetry of Kc
__global__ void k_class_dcondense(int ncls, const int* __restrict__ clsPset, const double* __restrict__ clsH,
                                  const double* __restrict__ psetM, const double* __restrict__ psetdM, const double* __restrict__ clsF33,
                                  const double* __restrict__ clsdF33, const int* __restrict__ clsBorn, double* __restrict__ dKc,
                                  double* __restrict__ dFc) {
  extern __shared__ double smd[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int cls = blockIdx.x * (blockDim.x >> 5) + warp;
  if (cls >= ncls) return;
  double* K = smd + warp * 2560;       // 1089
  double* dK = K + 1089;               // 1089
  double* Kaa = dK + 1089;             // 81
  double* X = Kaa + 81;                // 216 (9 x 24)
  double* y = X + 216;                 // 9
  double* t = y + 9;                   // 24
  const double hx = clsH[3 * cls], hy = clsH[3 * cls + 1], hz = clsH[3 * cls + 2];
  const double V8 = hx * hy * hz / 8;
  const double c0 = V8 * 4 / (hx * hx), c1 = V8 * 4 / (hy * hy), c2 = V8 * 4 / (hz * hz);
  const double c3 = V8 * 4 / (hx * hy), c4 = V8 * 4 / (hy * hz), c5 = V8 * 4 / (hz * hx);
  const double* M = psetM + (size_t)clsPset[cls] * 6 * 1089;
  const double* dM = psetdM + (size_t)clsPset[cls] * 6 * 1089;
  for (int o = lane; o < 1089; o += 32) {
    const int i = o / 33, j = o % 33;
    if (j >= i) {
      K[o] = c0 * M[o] + c1 * M[1089 + o] + c2 * M[2178 + o] + c3 * M[3267 + o] + c4 * M[4356 + o] + c5 * M[5445 + o];
      dK[o] = c0 * dM[o] + c1 * dM[1089 + o] + c2 * dM[2178 + o] + c3 * dM[3267 + o] + c4 * dM[4356 + o] + c5 * dM[5445 + o];
    }
  }
  __syncwarp();
  for (int o = lane; o < 1089; o += 32) {
    const int i = o / 33, j = o % 33;
    if (j < i) { K[o] = K[j * 33 + i]; dK[o] = dK[j * 33 + i]; }
  }
  __syncwarp();
  if (lane == 0) {
    for (int i = 0; i < 9; i++)
      for (int j = 0; j < 9; j++) Kaa[i * 9 + j] = K[(24 + i) * 33 + 24 + j];
    chol_dense9(Kaa, 1e-14);
  }
  __syncwarp();
  if (lane < 24) {
    double col[9];
    for (int i = 0; i < 9; i++) col[i] = K[(24 + i) * 33 + lane];
    chol_solve9(Kaa, col);
    for (int i = 0; i < 9; i++) X[i * 24 + lane] = col[i];
  }
  const bool born = clsBorn[cls] != 0;
  const double* f = clsF33 + (size_t)cls * 33;
  const double* df = clsdF33 + (size_t)cls * 33;
  if (lane == 0) {
    for (int i = 0; i < 9; i++) y[i] = born ? f[24 + i] : 0.0;
    chol_solve9(Kaa, y);
  }
  __syncwarp();
  // dKc = dKuu - dKua X - X^T dKau + X^T dKaa X
  double* out = dKc + (size_t)cls * 576;
  for (int e = lane; e < 576; e += 32) {
    const int i = e / 24, j = e % 24;
    double v = dK[i * 33 + j];
    for (int q = 0; q < 9; q++) v -= dK[i * 33 + 24 + q] * X[q * 24 + j] + X[q * 24 + i] * dK[(24 + q) * 33 + j];
    for (int q = 0; q < 9; q++) {
      double s2 = 0;
      for (int r = 0; r < 9; r++) s2 += dK[(24 + q) * 33 + 24 + r] * X[r * 24 + j];
      v += X[q * 24 + i] * s2;
    }
    out[e] = v;
  }
  __syncwarp();
  for (int e = lane; e < 576; e += 32) {
    const int i = e / 24, j = e % 24;
    if (j > i) {
      const double v = 0.5 * (out[i * 24 + j] + out[j * 24 + i]);
      out[i * 24 + j] = v;
      out[j * 24 + i] = v;
    }
  }
  // dfc = dfu - dKua y - X^T dfa + X^T dKaa y
  if (lane < 9) {
    double s2 = 0;
    for (int r = 0; r < 9; r++) s2 += dK[(24 + lane) * 33 + 24 + r] * y[r];
    t[lane] = s2 - (born ? df[24 + lane] : 0.0);   // dKaa y - dfa
  }
  __syncwarp();
  if (lane < 24) {
    double v = born ? df[lane] : 0.0;
    for (int q = 0; q < 9; q++) v -= dK[lane * 33 + 24 + q] * y[q];
    for (int q = 0; q < 9; q++) v += X[q * 24 + lane] * t[q];
    dFc[(size_t)cls * 24 + lane] = v;
  }
}

__device__ __forceinline__ int loc_index(int a, int b, int c) {
  // local node order loc of 06-mesher.js:49 -> index
  return c * 4 + (b ? (a ? 2 : 3) : (a ? 1 : 0));
}

// ---- stencil assembly: thread per (slot, node), contributions in element order -----------------
__global__ void k_assemble(int nn, int S, int nx, int ny, int nz, const int* __restrict__ posNode, const int* __restrict__ nodeIJK,
                           const int* __restrict__ nbr, const int* __restrict__ cellElems, const int* __restrict__ eClass,
                           const double* __restrict__ eScale, const int* __restrict__ eGroup, const int* __restrict__ groupStage, int stage,
                           int moduleStage, const double* __restrict__ clsKc, double* __restrict__ val) {
  const size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (t >= (size_t)NSLOT * S) return;
  const int s = (int)(t / S), ps = (int)(t % S);
  if (ps >= nn) {   // padding of the rows: zeros
    for (int v = 0; v < 9; v++) val[((size_t)s * 9 + v) * S + ps] = 0;
    return;
  }
  const int n = posNode[ps];
  double acc[9];
  for (int v = 0; v < 9; v++) acc[v] = 0;
  const int m = nbr[t];
  if (m >= 0) {
    const int i = nodeIJK[3 * n], j = nodeIJK[3 * n + 1], k = nodeIJK[3 * n + 2];
    const int di = s / 9 - 1, dj = (s / 3) % 3 - 1, dk = s % 3 - 1;
    const int ncy = ny - 1, ncz = nz - 1;
    const int ci0 = max(max(i, i + di) - 1, 0), ci1 = min(min(i, i + di), nx - 2);
    const int cj0 = max(max(j, j + dj) - 1, 0), cj1 = min(min(j, j + dj), ny - 2);
    const int ck0 = max(max(k, k + dk) - 1, 0), ck1 = min(min(k, k + dk), nz - 2);
    for (int ci = ci0; ci <= ci1; ci++)
      for (int cj = cj0; cj <= cj1; cj++)
        for (int ck = ck0; ck <= ck1; ck++) {
          const size_t cell = ((size_t)ci * ncy + cj) * ncz + ck;
          const int a = loc_index(i - ci, j - cj, k - ck), b = loc_index(i + di - ci, j + dj - cj, k + dk - ck);
          for (int q = 0; q < 2; q++) {
            const int e = cellElems[2 * cell + q];
            if (e < 0) continue;
            const bool born = groupStage[eGroup[e]] <= stage;
            if (moduleStage && !born) continue;   // module stages assemble the born parts only
            const double scale = eScale[e] * (born ? 1.0 : 1e-6);
            const double* Kc = clsKc + (size_t)eClass[e] * 576;
            for (int p = 0; p < 3; p++) {
              const int r = (3 * a + p) * 24 + 3 * b;
              acc[3 * p] += scale * Kc[r];
              acc[3 * p + 1] += scale * Kc[r + 1];
              acc[3 * p + 2] += scale * Kc[r + 2];
            }
          }
        }
  }
  for (int v = 0; v < 9; v++) val[((size_t)s * 9 + v) * S + ps] = acc[v];
}

// thermal load, thread per node (assembleStep's rhs, 09-assembly.js:417-420)
__global__ void k_assemble_rhs(int nn, int nx, int ny, int nz, const int* __restrict__ nodeIJK, const int* __restrict__ cellElems,
                               const int* __restrict__ eClass, const double* __restrict__ eScale, const int* __restrict__ eGroup,
                               const int* __restrict__ groupStage, int stage, int moduleStage, const int* __restrict__ clsBorn,
                               const double* __restrict__ clsFc, double* __restrict__ rhs) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= nn) return;
  const int i = nodeIJK[3 * n], j = nodeIJK[3 * n + 1], k = nodeIJK[3 * n + 2];
  const int ncy = ny - 1, ncz = nz - 1;
  double acc0 = 0, acc1 = 0, acc2 = 0;
  for (int ci = max(i - 1, 0); ci <= min(i, nx - 2); ci++)
    for (int cj = max(j - 1, 0); cj <= min(j, ny - 2); cj++)
      for (int ck = max(k - 1, 0); ck <= min(k, nz - 2); ck++) {
        const size_t cell = ((size_t)ci * ncy + cj) * ncz + ck;
        const int a = loc_index(i - ci, j - cj, k - ck);
        for (int q = 0; q < 2; q++) {
          const int e = cellElems[2 * cell + q];
          if (e < 0) continue;
          const int cls = eClass[e];
          if (!clsBorn[cls]) continue;
          const bool born = groupStage[eGroup[e]] <= stage;
          if (moduleStage && !born) continue;
          const double scale = eScale[e] * (born ? 1.0 : 1e-6);
          const double* fc = clsFc + (size_t)cls * 24;
          acc0 += scale * fc[3 * a];
          acc1 += scale * fc[3 * a + 1];
          acc2 += scale * fc[3 * a + 2];
        }
      }
  rhs[3 * n] = acc0; rhs[3 * n + 1] = acc1; rhs[3 * n + 2] = acc2;
}

// applyConstraints (09-assembly.js:445-464), thread per constrained DOF (nn: the row stride of the
// slot-major arrays). The reference walks the DOFs in order, but the result does not depend on
// the order: a DOF's row and column entries off the diagonal are set to zero (by every DOF that
// reaches them, all writing the same zero), and its diagonal, which no other DOF writes, is set to
// one only if it is zero.
__global__ void k_constraints(int nn, int ncon, const int* __restrict__ dofs, const int* __restrict__ pos, const int* __restrict__ nbr,
                              const int* __restrict__ slotMask, double* __restrict__ val, double* __restrict__ rhs,
                              uint8_t* __restrict__ isC) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= ncon) return;
  {
    const int d = dofs[t], i = d / 3, p = d % 3, pi = pos[i];
    isC[d] = 1;
    const int mask = slotMask[i];
    for (int s = 0; s < NSLOT; s++) {
      if (!(mask >> s & 1)) continue;
      const int j = nbr[(size_t)s * nn + pi];
      for (int q = 0; q < 3; q++) {
        double* v = val + ((size_t)s * 9 + 3 * p + q) * nn + pi;
        if (3 * j + q != d) *v = 0;
        else if (*v == 0) *v = 1;
      }
      const int s2 = NSLOT - 1 - s;
      for (int q = 0; q < 3; q++)
        if (3 * j + q != d) val[((size_t)s2 * 9 + 3 * q + p) * nn + pos[j]] = 0;
    }
    if (rhs) rhs[d] = 0;
  }
}

// _scale (10-solver.js:852-866)
__global__ void k_scale_diag(int nn, int S, const int* __restrict__ posNode, const double* __restrict__ val, double* __restrict__ s) {
  const int ps = blockIdx.x * blockDim.x + threadIdx.x;
  if (ps >= nn) return;
  const int n = posNode[ps];
  for (int p = 0; p < 3; p++) s[3 * n + p] = 1 / sqrt(fmax(val[((size_t)SLOT_SELF * 9 + 4 * p) * S + ps], 1e-300));
}

__global__ void k_scale_val(int nn, int S, const int* __restrict__ posNode, const int* __restrict__ nbr, const double* __restrict__ s,
                            double* __restrict__ val) {
  const size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (t >= (size_t)NSLOT * nn) return;
  const int sl = (int)(t / nn), ps = (int)(t % nn), n = posNode[ps];
  const int j = nbr[(size_t)sl * S + ps];
  if (j < 0) return;
  for (int p = 0; p < 3; p++)
    for (int q = 0; q < 3; q++) {
      double* v = val + ((size_t)sl * 9 + 3 * p + q) * S + ps;
      *v *= s[3 * n + p] * s[3 * j + q];
    }
}

__global__ void k_mul(size_t n, const double* __restrict__ a, const double* __restrict__ b, double* __restrict__ y) {
  const size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (i < n) y[i] = a[i] * b[i];
}

// chol3 (10-solver.js:12-25)
__device__ bool chol3(const double* A, double* L, double jit) {
  const double a00 = A[0] + jit, a10 = A[3], a11 = A[4] + jit, a20 = A[6], a21 = A[7], a22 = A[8] + jit;
  if (!(a00 > 0)) return false;
  const double l00 = sqrt(a00);
  const double l10 = a10 / l00, l20 = a20 / l00;
  const double d11 = a11 - l10 * l10;
  if (!(d11 > 0)) return false;
  const double l11 = sqrt(d11);
  const double l21 = (a21 - l20 * l10) / l11;
  const double d22 = a22 - l20 * l20 - l21 * l21;
  if (!(d22 > 0)) return false;
  L[0] = l00; L[1] = 0; L[2] = 0; L[3] = l10; L[4] = l11; L[5] = 0; L[6] = l20; L[7] = l21; L[8] = sqrt(d22);
  return true;
}

// factorColumns (10-solver.js:31-68), thread per column (nn: the row stride of the slot-major
// arrays)
__global__ void k_factor_columns(int ncol, int nn, const int* __restrict__ colStart, const int* __restrict__ pos, const int* __restrict__ nbr,
                                 const int* __restrict__ slotMask, const double* __restrict__ val, double* __restrict__ F,
                                 int* __restrict__ jitterCount) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ncol) return;
  int jitter = 0;
  double D[9], tmp[9];
  const int p0 = colStart[c] < colStart[c + 1] ? pos[colStart[c]] : 0;
  for (int n = colStart[c]; n < colStart[c + 1]; n++) {
    const int pn = p0 + (n - colStart[c]);
    for (int q = 0; q < 9; q++) D[q] = val[((size_t)SLOT_SELF * 9 + q) * nn + pn];
    double* Fn = F + 18 * (size_t)pn;
    const bool down = n > colStart[c] && (slotMask[n] >> SLOT_DOWN & 1) && nbr[(size_t)SLOT_DOWN * nn + pn] == n - 1;
    if (down) {
      const double* Fp = F + 18 * (size_t)(pn - 1);
      for (int r = 0; r < 3; r++) {
        const double b0 = val[((size_t)SLOT_DOWN * 9 + 3 * r) * nn + pn], b1 = val[((size_t)SLOT_DOWN * 9 + 3 * r + 1) * nn + pn],
                     b2 = val[((size_t)SLOT_DOWN * 9 + 3 * r + 2) * nn + pn];
        const double y0 = b0 / Fp[0];
        const double y1 = (b1 - Fp[3] * y0) / Fp[4];
        const double y2 = (b2 - Fp[6] * y0 - Fp[7] * y1) / Fp[8];
        tmp[3 * r] = y0; tmp[3 * r + 1] = y1; tmp[3 * r + 2] = y2;
      }
      for (int q = 0; q < 9; q++) Fn[9 + q] = tmp[q];
      for (int r = 0; r < 3; r++)
        for (int cc = 0; cc < 3; cc++)
          D[3 * r + cc] -= tmp[3 * r] * tmp[3 * cc] + tmp[3 * r + 1] * tmp[3 * cc + 1] + tmp[3 * r + 2] * tmp[3 * cc + 2];
    } else {
      for (int q = 0; q < 9; q++) Fn[9 + q] = 0;
    }
    double jit = 0;
    for (int t = 0; t < 8 && !chol3(D, Fn, jit); t++) {
      jit = jit != 0 ? jit * 10 : 1e-10 * fmax(fmax(fabs(D[0]), fabs(D[4])), fmax(fabs(D[8]), 1e-300));
      jitter++;
    }
    // reciprocal pivots in the upper slots of the lower factor (always 0 in L): the smoother
    // multiplies by them instead of dividing; the factorisation itself never reads these slots
    Fn[1] = 1 / Fn[0];
    Fn[2] = 1 / Fn[4];
    Fn[5] = 1 / Fn[8];
  }
  if (jitter) atomicAdd(jitterCount, jitter);
}

// shellWeights (10-solver.js:337-353): 3x6 weights per node with the scaling folded in
__global__ void k_w01(int nn, const double* __restrict__ s, const double* __restrict__ zp, double* __restrict__ W) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= nn) return;
  double* w = W + 18 * (size_t)n;
  for (int q = 0; q < 18; q++) w[q] = 0;
  const double z = zp[n];
  w[0] = 1 / s[3 * n]; w[4] = z / s[3 * n];
  w[7] = 1 / s[3 * n + 1]; w[9] = -z / s[3 * n + 1];
  w[14] = 1 / s[3 * n + 2]; w[17] = z / s[3 * n + 2];
}


// factorShellColumns (10-solver.js:474-494) with cholDense (rel 1e-12), warp per column
__global__ void k_factor_shell(int ncol, const int* __restrict__ colStart, const int* __restrict__ rowPtr, const int* __restrict__ col,
                               const double* __restrict__ val, const long long* __restrict__ cfPtr, double* __restrict__ cf,
                               int* __restrict__ jitterCount) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int c = blockIdx.x * (blockDim.x >> 5) + warp;
  if (c >= ncol) return;
  const int n0 = colStart[c], n1 = colStart[c + 1], m = (n1 - n0) * 6;
  if (!m) return;
  double* A = cf + cfPtr[c];
  for (int e = lane; e < m * m; e += 32) A[e] = 0;
  __syncwarp();
  for (int n = n0; n < n1; n++)
    for (int k = rowPtr[n]; k < rowPtr[n + 1]; k++) {
      const int j = col[k];
      if (j < n0 || j >= n1) continue;
      for (int e = lane; e < 36; e += 32) {
        const int p = e / 6, q = e % 6;
        A[((n - n0) * 6 + p) * m + (j - n0) * 6 + q] = val[36 * (size_t)k + e];
      }
    }
  __syncwarp();
  double dmax = 0;
  for (int i = 0; i < m; i++) dmax = fmax(dmax, fabs(A[i * m + i]));
  const double jitter = 1e-12 * (dmax != 0 ? dmax : 1);
  int fixes = 0;
  for (int j = 0; j < m; j++) {
    const int rj = j * m;
    double inv = 0;
    if (lane == 0) {
      double d = A[rj + j];
      for (int k = 0; k < j; k++) d -= A[rj + k] * A[rj + k];
      if (!(d > jitter)) { d = fmax(fabs(d), jitter); fixes++; }
      const double ljj = sqrt(d);
      A[rj + j] = ljj;
      inv = 1 / ljj;
    }
    inv = __shfl_sync(0xffffffffu, inv, 0);
    __syncwarp();
    for (int i = j + 1 + lane; i < m; i += 32) {
      const int ri = i * m;
      double s = A[ri + j];
      for (int k = 0; k < j; k++) s -= A[ri + k] * A[rj + k];
      A[ri + j] = s * inv;
    }
    __syncwarp();
  }
  if (lane == 0 && fixes) atomicAdd(jitterCount, fixes);
}

// explicit inverse of every shell column block from its Cholesky factor (warp per column, lanes over
// unit vectors); the smoother then applies A_cc^-1 as a dense product instead of two serial
// triangular solves (cholSolveDenseOff, 10-solver.js:497-509, computes the same A_cc^-1 r).
// Column e of the inverse is stored contiguously (entry (i, e) at e*m + i), so that the lanes of
// the smoother, one per row e, read entry (e, k) at k*m + e with coalesced loads.
__global__ void k_shell_inverse(int ncol, const int* __restrict__ colStart, const long long* __restrict__ cfPtr,
                                const double* __restrict__ cf, double* __restrict__ cfInv) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int c = blockIdx.x * (blockDim.x >> 5) + warp;
  if (c >= ncol) return;
  const int m = 6 * (colStart[c + 1] - colStart[c]);
  if (!m) return;
  const double* L = cf + cfPtr[c];
  for (int e = lane; e < m; e += 32) {
    double* Xe = cfInv + cfPtr[c] + (size_t)e * m;
    for (int i = 0; i < m; i++) {
      double s = i == e ? 1.0 : 0.0;
      for (int k = e; k < i; k++) s -= L[i * m + k] * Xe[k];
      Xe[i] = i < e ? 0.0 : s / L[i * m + i];
    }
    for (int i = m - 1; i >= 0; i--) {
      double s = Xe[i];
      for (int k = i + 1; k < m; k++) s -= L[k * m + i] * Xe[k];
      Xe[i] = s / L[i * m + i];
    }
  }
}

__global__ void k_to_f32(size_t n, const double* __restrict__ a, float* __restrict__ b) {
  const size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (i < n) b[i] = (float)a[i];
}

// ---- element DOF histories at screening sites -----------------------------------------------
// natural coordinates of the 8 nodes in the local order of the mesher (06-mesher.js:49)
__device__ __forceinline__ double node_xi(int a) { return ((a & 3) == 1 || (a & 3) == 2) ? 1.0 : -1.0; }
__device__ __forceinline__ double node_eta(int a) { return (a & 3) >= 2 ? 1.0 : -1.0; }
__device__ __forceinline__ double node_zeta(int a) { return a >= 4 ? 1.0 : -1.0; }

// Model.accumulateStep with qOnly (09-assembly.js:508-533), one warp per listed element:
// q[33 t ..] += (du at the element's nodes, K_aa^-1 (f_a - K_au du)) with K_a. the rows 24..32 of
// the step's K33 = sum_m c_m M^m taken as stored (stepRecovery, 09-assembly.js:480-491) and f_a
// the incompatible-mode part of the element thermal load of a born material. Same operations in
// the same order as the reference, so q matches it bit for bit for the same du.
__global__ void k_accumulate_q(int nel, int ne, const int* __restrict__ elems, const int* __restrict__ conn,
                               const int* __restrict__ eClass, const int* __restrict__ clsPset,
                               const double* __restrict__ clsH, const double* __restrict__ psetM,
                               const double* __restrict__ clsF33, const double* __restrict__ du,
                               double* __restrict__ q) {
  __shared__ double sm[4][448];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int t = blockIdx.x * 4 + warp;
  if (t >= nel) return;
  double* Kr = sm[warp];               // 297
  double* Kaa = Kr + 297;              // 81
  double* dq = Kaa + 81;               // 24
  double* col = dq + 24;               // 9
  const int e = elems[t];
  if (e < 0 || e >= ne) {              // no element at this site: its DOFs read NaN
    for (int o = lane; o < 33; o += 32) q[33 * (size_t)t + o] = CUDART_NAN;
    return;
  }
  const int cls = eClass[e];
  const double hx = clsH[3 * cls], hy = clsH[3 * cls + 1], hz = clsH[3 * cls + 2];
  const double V8 = hx * hy * hz / 8;
  const double c0 = V8 * 4 / (hx * hx), c1 = V8 * 4 / (hy * hy), c2 = V8 * 4 / (hz * hz);
  const double c3 = V8 * 4 / (hx * hy), c4 = V8 * 4 / (hy * hz), c5 = V8 * 4 / (hz * hx);
  const double* Ma = psetM + (size_t)clsPset[cls] * 6 * 1089 + 24 * 33;
  for (int r = lane; r < 297; r += 32)
    Kr[r] = c0 * Ma[r] + c1 * Ma[1089 + r] + c2 * Ma[2178 + r] + c3 * Ma[3267 + r] + c4 * Ma[4356 + r] + c5 * Ma[5445 + r];
  if (lane < 24) dq[lane] = du[3 * (size_t)conn[8 * (size_t)e + lane / 3] + lane % 3];
  __syncwarp();
  for (int o = lane; o < 81; o += 32) Kaa[o] = Kr[(o / 9) * 33 + 24 + o % 9];
  if (lane < 9) {
    double s = clsF33[(size_t)cls * 33 + 24 + lane];
    for (int k = 0; k < 24; k++) s -= Kr[lane * 33 + k] * dq[k];
    col[lane] = s;
  }
  __syncwarp();
  if (lane == 0) {
    chol_dense9(Kaa, 1e-14);
    chol_solve9(Kaa, col);
  }
  __syncwarp();
  for (int o = lane; o < 33; o += 32) q[33 * (size_t)t + o] += o < 24 ? dq[o] : col[o - 24];
}

// Model.accumulateStep without qOnly (09-assembly.js:508-544), warp per listed element: the DOF
// increment as in k_accumulate_q, state[0..32] += dq and, when the material is born, the strain
// polynomial E of dq (boxStrainPoly, :176-196) and per sub-layer S_m += D_m E_m (m < 7) and
// S_th += the step's thermal stress increment (homogeneous sets: one layer with the set's D, s0)
__global__ void k_accumulate_state(int nel, int ne, const int* __restrict__ elems, const int* __restrict__ conn,
                                   const int* __restrict__ eClass, const int* __restrict__ clsPset, const double* __restrict__ clsH,
                                   const double* __restrict__ psetM, const double* __restrict__ clsF33, const int* __restrict__ clsBorn,
                                   const int* __restrict__ psetLayered, const double* __restrict__ stepD, const double* __restrict__ stepS0,
                                   const int* __restrict__ subOff, const double* __restrict__ subD, const double* __restrict__ subS0,
                                   const double* __restrict__ du, int stride, double* __restrict__ state) {
  __shared__ double sm[4][448];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int t = blockIdx.x * 4 + warp;
  if (t >= nel) return;
  double* Kr = sm[warp];               // 297 (then the strain polynomial, 42)
  double* Kaa = Kr + 297;              // 81
  double* dq = Kaa + 81;               // 33: nodal DOFs, then the incompatible modes
  double* st = state + (size_t)stride * t;
  const int e = elems[t];
  if (e < 0 || e >= ne) {
    for (int o = lane; o < stride; o += 32) st[o] = CUDART_NAN;
    return;
  }
  const int cls = eClass[e];
  const double hx = clsH[3 * cls], hy = clsH[3 * cls + 1], hz = clsH[3 * cls + 2];
  const double V8 = hx * hy * hz / 8;
  const double c0 = V8 * 4 / (hx * hx), c1 = V8 * 4 / (hy * hy), c2 = V8 * 4 / (hz * hz);
  const double c3 = V8 * 4 / (hx * hy), c4 = V8 * 4 / (hy * hz), c5 = V8 * 4 / (hz * hx);
  const int pset = clsPset[cls];
  const double* Ma = psetM + (size_t)pset * 6 * 1089 + 24 * 33;
  for (int r = lane; r < 297; r += 32)
    Kr[r] = c0 * Ma[r] + c1 * Ma[1089 + r] + c2 * Ma[2178 + r] + c3 * Ma[3267 + r] + c4 * Ma[4356 + r] + c5 * Ma[5445 + r];
  if (lane < 24) dq[lane] = du[3 * (size_t)conn[8 * (size_t)e + lane / 3] + lane % 3];
  __syncwarp();
  for (int o = lane; o < 81; o += 32) Kaa[o] = Kr[(o / 9) * 33 + 24 + o % 9];
  if (lane < 9) {
    double s = clsF33[(size_t)cls * 33 + 24 + lane];
    for (int k = 0; k < 24; k++) s -= Kr[lane * 33 + k] * dq[k];
    dq[24 + lane] = s;
  }
  __syncwarp();
  if (lane == 0) {
    chol_dense9(Kaa, 1e-14);
    chol_solve9(Kaa, dq + 24);
  }
  __syncwarp();
  for (int o = lane; o < 33; o += 32) st[o] += dq[o];
  if (!clsBorn[cls]) return;
  double* E = Kr;
  if (lane == 0) {
    for (int q = 0; q < 42; q++) E[q] = 0;
    const double sx = 2 / hx, sy = 2 / hy, sz = 2 / hz;
    for (int a = 0; a < 8; a++) {
      const double xa = node_xi(a), ya = node_eta(a), za = node_zeta(a);
      const double ux = dq[3 * a], uy = dq[3 * a + 1], uz = dq[3 * a + 2];
      const double cx = xa * sx / 8, cy = ya * sy / 8, cz = za * sz / 8;
      const int mx[4] = {0, 2, 3, 5}, my[4] = {0, 1, 3, 6}, mz[4] = {0, 1, 2, 4};
      const double vx[4] = {cx, cx * ya, cx * za, cx * ya * za}, vy[4] = {cy, cy * xa, cy * za, cy * xa * za},
                   vz[4] = {cz, cz * xa, cz * ya, cz * xa * ya};
      for (int k = 0; k < 4; k++) { const int m = mx[k]; const double c = vx[k]; E[6 * m] += c * ux; E[6 * m + 3] += c * uy; E[6 * m + 5] += c * uz; }
      for (int k = 0; k < 4; k++) { const int m = my[k]; const double c = vy[k]; E[6 * m + 1] += c * uy; E[6 * m + 3] += c * ux; E[6 * m + 4] += c * uz; }
      for (int k = 0; k < 4; k++) { const int m = mz[k]; const double c = vz[k]; E[6 * m + 2] += c * uz; E[6 * m + 4] += c * uy; E[6 * m + 5] += c * ux; }
    }
    const double* a1 = dq + 24; const double* a2 = dq + 27; const double* a3 = dq + 30;
    E[6] += -2 * sx * a1[0]; E[6 + 3] += -2 * sx * a1[1]; E[6 + 5] += -2 * sx * a1[2];
    E[12 + 1] += -2 * sy * a2[1]; E[12 + 3] += -2 * sy * a2[0]; E[12 + 4] += -2 * sy * a2[2];
    E[18 + 2] += -2 * sz * a3[2]; E[18 + 4] += -2 * sz * a3[1]; E[18 + 5] += -2 * sz * a3[0];
  }
  __syncwarp();
  const bool lay = psetLayered[pset] != 0;
  const int ns = lay ? subOff[pset + 1] - subOff[pset] : 1;
  for (int idx = lane; idx < 48 * ns; idx += 32) {
    const int s = idx / 48, rem = idx % 48;
    const double* D = lay ? subD + 36 * (size_t)(subOff[pset] + s) : stepD + 36 * (size_t)pset;
    const double* s0 = lay ? subS0 + 6 * (size_t)(subOff[pset] + s) : stepS0 + 6 * (size_t)pset;
    double* o = st + 33 + 48 * s;
    if (rem < 42) {
      const int mo = rem / 6, r = rem % 6;
      double v = 0;
      for (int k = 0; k < 6; k++) v += D[r * 6 + k] * E[6 * mo + k];
      o[6 * mo + r] += v;
    } else {
      o[rem] += s0[rem - 42];
    }
  }
}

// stateStress (09-assembly.js:555-571) with subLayerAt (:547-552), thread per point: total strain
// and stress of element elem[t] from its state at the natural point nat[3 t ..]
__global__ void k_state_stress(int np, int ne, const int* __restrict__ elem, const int* __restrict__ eClass,
                               const int* __restrict__ clsPset, const double* __restrict__ clsH, const int* __restrict__ eIJK,
                               const double* __restrict__ zs, const int* __restrict__ psetLayered, const int* __restrict__ subOff,
                               const double* __restrict__ subZ, const double* __restrict__ state, int stride,
                               const double* __restrict__ nat, double* __restrict__ eps, double* __restrict__ sig) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= np) return;
  double* oe = eps + 6 * (size_t)t;
  double* os = sig + 6 * (size_t)t;
  const int e = elem[t];
  if (e < 0 || e >= ne) {
    for (int r = 0; r < 6; r++) { oe[r] = CUDART_NAN; os[r] = CUDART_NAN; }
    return;
  }
  const int cls = eClass[e];
  const double sx = 2 / clsH[3 * cls], sy = 2 / clsH[3 * cls + 1], sz = 2 / clsH[3 * cls + 2];
  const double xi = nat[3 * (size_t)t], eta = nat[3 * (size_t)t + 1], zeta = nat[3 * (size_t)t + 2];
  const double* u = state + (size_t)stride * t;
  double e0 = 0, e1 = 0, e2 = 0, e3 = 0, e4 = 0, e5 = 0;
  for (int b = 0; b < 11; b++) {
    double dx, dy, dz;
    if (b < 8) {
      const double xa = node_xi(b), ya = node_eta(b), za = node_zeta(b);
      dx = xa * (1 + ya * eta) * (1 + za * zeta) * 0.125 * sx;
      dy = ya * (1 + xa * xi) * (1 + za * zeta) * 0.125 * sy;
      dz = za * (1 + xa * xi) * (1 + ya * eta) * 0.125 * sz;
    } else {
      dx = b == 8 ? -2 * xi * sx : 0;
      dy = b == 9 ? -2 * eta * sy : 0;
      dz = b == 10 ? -2 * zeta * sz : 0;
    }
    const double ux = u[3 * b], uy = u[3 * b + 1], uz = u[3 * b + 2];
    e0 += dx * ux; e1 += dy * uy; e2 += dz * uz;
    e3 += dy * ux + dx * uy;
    e4 += dz * uy + dy * uz;
    e5 += dz * ux + dx * uz;
  }
  oe[0] = e0; oe[1] = e1; oe[2] = e2; oe[3] = e3; oe[4] = e4; oe[5] = e5;
  const int pset = clsPset[cls];
  int s = 0;
  if (psetLayered[pset]) {
    const int k = eIJK[3 * (size_t)e + 2];
    const double z = zs[k] + 0.5 * (zeta + 1) * (zs[k + 1] - zs[k]);
    const int ns = subOff[pset + 1] - subOff[pset];
    s = ns - 1;
    for (int q = 0; q < ns; q++)
      if (z <= subZ[2 * (size_t)(subOff[pset] + q) + 1] + 1e-12) { s = q; break; }
  }
  const double phi[7] = {1, xi, eta, zeta, xi * eta, eta * zeta, xi * zeta};
  const double* o = u + 33 + 48 * s;
  for (int r = 0; r < 6; r++) {
    double v = -o[42 + r];
    for (int mo = 0; mo < 7; mo++) v += phi[mo] * o[6 * mo + r];
    os[r] = v;
  }
}

// ---- adjoint sensitivities of a warpage measure -------------------------------------------------
// per element e (warp per element): with s_e its assembly scale (eScale, 1e-6 before its stage),
// out[2e] = s_e lambda_e^T Kc u_e and out[2e+1] = s_e lambda_e^T fc, from the condensed class
// matrix and load of the step assembled last (lanes over the 24 rows, fixed-order warp sum)
__global__ void k_sens_elements(int ne, const int* __restrict__ conn, const int* __restrict__ eClass, const double* __restrict__ eScale,
                                const int* __restrict__ eGroup, const int* __restrict__ groupStage, int stage,
                                const double* __restrict__ clsKc, const double* __restrict__ clsFc, const double* __restrict__ u,
                                const double* __restrict__ lam, double* __restrict__ out) {
  __shared__ double su[4][24];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int e = blockIdx.x * 4 + warp;
  if (e >= ne) return;
  const int cls = eClass[e];
  double lk = 0;
  if (lane < 24) {
    const size_t dof = 3 * (size_t)conn[8 * (size_t)e + lane / 3] + lane % 3;
    su[warp][lane] = u[dof];
    lk = lam[dof];
  }
  __syncwarp();
  double t1 = 0, t2 = 0;
  if (lane < 24) {
    const double* K = clsKc + 576 * (size_t)cls + 24 * lane;
    double ku = 0;
    for (int b = 0; b < 24; b++) ku += K[b] * su[warp][b];
    t1 = lk * ku;
    t2 = lk * clsFc[24 * (size_t)cls + lane];
  }
  for (int off = 16; off > 0; off >>= 1) {
    t1 += __shfl_xor_sync(0xffffffffu, t1, off);
    t2 += __shfl_xor_sync(0xffffffffu, t2, off);
  }
  if (lane == 0) {
    const double sc = eScale[e] * (groupStage[eGroup[e]] <= stage ? 1.0 : 1e-6);
    out[2 * (size_t)e] = sc * t1;
    out[2 * (size_t)e + 1] = sc * t2;
  }
}

// per property set sums of the element terms, in a fixed order: block b sums elements
// b*chunk .. (b+1)*chunk-1 per set (thread-strided, then a tree per set), one partial per block
constexpr int SENS_MAXSET = 64;
__global__ void __launch_bounds__(256) k_sens_partial(int ne, int chunk, const int* __restrict__ eClass, const int* __restrict__ clsPset,
                                                      int npset, const double* __restrict__ et, double* __restrict__ part) {
  __shared__ double s1[256], s2[256];
  const int e0 = blockIdx.x * chunk, e1 = min(ne, e0 + chunk);
  for (int p = 0; p < npset; p++) {
    double a = 0, b = 0;
    for (int e = e0 + threadIdx.x; e < e1; e += blockDim.x)
      if (clsPset[eClass[e]] == p) { a += et[2 * (size_t)e]; b += et[2 * (size_t)e + 1]; }
    s1[threadIdx.x] = a; s2[threadIdx.x] = b;
    __syncthreads();
    for (int h = 128; h > 0; h >>= 1) {
      if ((int)threadIdx.x < h) { s1[threadIdx.x] += s1[threadIdx.x + h]; s2[threadIdx.x] += s2[threadIdx.x + h]; }
      __syncthreads();
    }
    if (threadIdx.x == 0) { part[2 * ((size_t)blockIdx.x * npset + p)] = s1[0]; part[2 * ((size_t)blockIdx.x * npset + p) + 1] = s2[0]; }
    __syncthreads();
  }
}

// boxStrainAt (07-element.js:127-142) with boxDerivs (:19-30), thread per point: engineering
// strain of element elem[t] with DOFs q[33 t ..] at the natural point nat[3 t ..]
__global__ void k_element_strains(int np, int ne, const int* __restrict__ elem, const int* __restrict__ eClass,
                                  const double* __restrict__ clsH, const double* __restrict__ q,
                                  const double* __restrict__ nat, double* __restrict__ eps) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= np) return;
  double* o = eps + 6 * (size_t)t;
  const int e = elem[t];
  if (e < 0 || e >= ne) {
    for (int r = 0; r < 6; r++) o[r] = CUDART_NAN;
    return;
  }
  const int cls = eClass[e];
  const double sx = 2 / clsH[3 * cls], sy = 2 / clsH[3 * cls + 1], sz = 2 / clsH[3 * cls + 2];
  const double xi = nat[3 * (size_t)t], eta = nat[3 * (size_t)t + 1], zeta = nat[3 * (size_t)t + 2];
  const double* u = q + 33 * (size_t)t;
  double e0 = 0, e1 = 0, e2 = 0, e3 = 0, e4 = 0, e5 = 0;
  for (int b = 0; b < 11; b++) {
    double dx, dy, dz;
    if (b < 8) {
      const double xa = node_xi(b), ya = node_eta(b), za = node_zeta(b);
      dx = xa * (1 + ya * eta) * (1 + za * zeta) * 0.125 * sx;
      dy = ya * (1 + xa * xi) * (1 + za * zeta) * 0.125 * sy;
      dz = za * (1 + xa * xi) * (1 + ya * eta) * 0.125 * sz;
    } else {
      dx = b == 8 ? -2 * xi * sx : 0;
      dy = b == 9 ? -2 * eta * sy : 0;
      dz = b == 10 ? -2 * zeta * sz : 0;
    }
    const double ux = u[3 * b], uy = u[3 * b + 1], uz = u[3 * b + 2];
    e0 += dx * ux; e1 += dy * uy; e2 += dz * uz;
    e3 += dy * ux + dx * uy;
    e4 += dz * uy + dy * uz;
    e5 += dz * ux + dx * uz;
  }
  o[0] = e0; o[1] = e1; o[2] = e2; o[3] = e3; o[4] = e4; o[5] = e5;
}

// the transpose of boxStrainAt (07-element.js:127-142), thread per point: gq[33 t ..] = B(nat)^T
// g[6 t ..] with B the strain operator of k_element_strains (the derivative of a function of the
// strains with respect to the element DOFs)
__global__ void k_element_strains_adjoint(int np, int ne, const int* __restrict__ elem, const int* __restrict__ eClass,
                                          const double* __restrict__ clsH, const double* __restrict__ nat, const double* __restrict__ g,
                                          double* __restrict__ gq) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= np) return;
  double* o = gq + 33 * (size_t)t;
  const int e = elem[t];
  if (e < 0 || e >= ne) {
    for (int r = 0; r < 33; r++) o[r] = CUDART_NAN;
    return;
  }
  const int cls = eClass[e];
  const double sx = 2 / clsH[3 * cls], sy = 2 / clsH[3 * cls + 1], sz = 2 / clsH[3 * cls + 2];
  const double xi = nat[3 * (size_t)t], eta = nat[3 * (size_t)t + 1], zeta = nat[3 * (size_t)t + 2];
  const double* gv = g + 6 * (size_t)t;
  const double g0 = gv[0], g1 = gv[1], g2 = gv[2], g3 = gv[3], g4 = gv[4], g5 = gv[5];
  for (int b = 0; b < 11; b++) {
    double dx, dy, dz;
    if (b < 8) {
      const double xa = node_xi(b), ya = node_eta(b), za = node_zeta(b);
      dx = xa * (1 + ya * eta) * (1 + za * zeta) * 0.125 * sx;
      dy = ya * (1 + xa * xi) * (1 + za * zeta) * 0.125 * sy;
      dz = za * (1 + xa * xi) * (1 + ya * eta) * 0.125 * sz;
    } else {
      dx = b == 8 ? -2 * xi * sx : 0;
      dy = b == 9 ? -2 * eta * sy : 0;
      dz = b == 10 ? -2 * zeta * sz : 0;
    }
    o[3 * b] = dx * g0 + dy * g3 + dz * g5;
    o[3 * b + 1] = dy * g1 + dx * g3 + dz * g4;
    o[3 * b + 2] = dz * g2 + dy * g4 + dx * g5;
  }
}

// the transpose of one step of k_accumulate_q, warp per listed element: with the step's
// q increment dq = (du_e, alpha), alpha = K_aa^-1 (f_a - K_au du_e), and gq (33) the derivative of
// a function with respect to dq, gdu (24) = gq_u - K_au^T K_aa^-1 gq_a is its derivative with
// respect to du_e, and gA = (K_aa^-1 gq_a)^T f_a its derivative with respect to the logarithm of the
// thermal strain of the element's property set through alpha (alpha does not change when the set's
// stiffness is scaled)
__global__ void k_accumulate_q_adjoint(int nel, int ne, const int* __restrict__ elems, const int* __restrict__ eClass,
                                       const int* __restrict__ clsPset, const double* __restrict__ clsH, const double* __restrict__ psetM,
                                       const double* __restrict__ clsF33, const double* __restrict__ gq, double* __restrict__ gdu,
                                       double* __restrict__ gA) {
  __shared__ double sm[4][420];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int t = blockIdx.x * 4 + warp;
  if (t >= nel) return;
  double* Kr = sm[warp];               // 297
  double* Kaa = Kr + 297;              // 81
  double* w = Kaa + 81;                // 9
  const int e = elems[t];
  if (e < 0 || e >= ne) {
    for (int o = lane; o < 24; o += 32) gdu[24 * (size_t)t + o] = CUDART_NAN;
    if (lane == 0) gA[t] = CUDART_NAN;
    return;
  }
  const int cls = eClass[e];
  const double hx = clsH[3 * cls], hy = clsH[3 * cls + 1], hz = clsH[3 * cls + 2];
  const double V8 = hx * hy * hz / 8;
  const double c0 = V8 * 4 / (hx * hx), c1 = V8 * 4 / (hy * hy), c2 = V8 * 4 / (hz * hz);
  const double c3 = V8 * 4 / (hx * hy), c4 = V8 * 4 / (hy * hz), c5 = V8 * 4 / (hz * hx);
  const double* Ma = psetM + (size_t)clsPset[cls] * 6 * 1089 + 24 * 33;
  for (int r = lane; r < 297; r += 32)
    Kr[r] = c0 * Ma[r] + c1 * Ma[1089 + r] + c2 * Ma[2178 + r] + c3 * Ma[3267 + r] + c4 * Ma[4356 + r] + c5 * Ma[5445 + r];
  if (lane < 9) w[lane] = gq[33 * (size_t)t + 24 + lane];
  __syncwarp();
  for (int o = lane; o < 81; o += 32) Kaa[o] = Kr[(o / 9) * 33 + 24 + o % 9];
  __syncwarp();
  if (lane == 0) {
    chol_dense9(Kaa, 1e-14);
    chol_solve9(Kaa, w);   // K_aa is symmetric: K_aa^-T gq_a = K_aa^-1 gq_a
  }
  __syncwarp();
  if (lane < 24) {
    double s = gq[33 * (size_t)t + lane];
    for (int r = 0; r < 9; r++) s -= Kr[r * 33 + lane] * w[r];
    gdu[24 * (size_t)t + lane] = s;
  }
  if (lane == 0) {
    double a = 0;
    for (int r = 0; r < 9; r++) a += w[r] * clsF33[(size_t)cls * 33 + 24 + r];
    gA[t] = a;
  }
}

// findInterval (01-util.js:12-22): i with a[i] <= x < a[i+1], clamped to [0, n-2]
__device__ int find_interval(const double* __restrict__ a, int n, double x) {
  if (x <= a[0]) return 0;
  if (x >= a[n - 1]) return n - 2;
  int lo = 0, hi = n - 1;
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (a[mid] <= x) lo = mid; else hi = mid;
  }
  return lo;
}

// samplePlane (12-post.js:30-38), thread per point: bilinear interpolation of component comp of
// the nodal field u on mesh plane k at (x, y); NaN where a corner node does not exist
__global__ void k_sample_plane(int npts, int nx, int ny, int nz, const double* __restrict__ xs, const double* __restrict__ ys,
                               const int* __restrict__ nodeId, const double* __restrict__ u, int k, int comp,
                               const double* __restrict__ px, const double* __restrict__ py, double* __restrict__ out) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= npts) return;
  const double x = px[t], y = py[t];
  const int i = find_interval(xs, nx, x), j = find_interval(ys, ny, y);
  const double tx = (x - xs[i]) / (xs[i + 1] - xs[i]), ty = (y - ys[j]) / (ys[j + 1] - ys[j]);
  const size_t r0 = ((size_t)i * ny + j) * nz + k, r1 = ((size_t)(i + 1) * ny + j) * nz + k;
  const int n00 = nodeId[r0], n10 = nodeId[r1], n01 = nodeId[r0 + nz], n11 = nodeId[r1 + nz];
  if (n00 < 0 || n10 < 0 || n01 < 0 || n11 < 0) {
    out[t] = CUDART_NAN;
    return;
  }
  out[t] = (1 - tx) * (1 - ty) * u[3 * (size_t)n00 + comp] + tx * (1 - ty) * u[3 * (size_t)n10 + comp] +
           (1 - tx) * ty * u[3 * (size_t)n01 + comp] + tx * ty * u[3 * (size_t)n11 + comp];
}

}  // namespace

void launch_shape_matrices(Context& c, const tm_step& st) {
  std::vector<double> M((size_t)c.npset * 6 * 1089);
  std::vector<int> lay(c.npset), born(c.npset);
  for (int p = 0; p < c.npset; p++) {
    lay[p] = st.psetLayered[p] != 0;
    born[p] = st.psetBorn[p] != 0;
    shape_matrices(lay[p] ? st.W + 108 * (size_t)p : nullptr, lay[p] ? nullptr : st.D + 36 * (size_t)p, M.data() + (size_t)p * 6 * 1089);
  }
  // element thermal loads per class (elementFth) on the host: a few hundred flops per class
  std::vector<double> f33((size_t)c.ncls * 33, 0.0);
  std::vector<int> clsBorn(c.ncls);
  for (int k = 0; k < c.ncls; k++) {
    const int p = c.clsPset[k];
    clsBorn[k] = born[p];
    if (!born[p]) continue;
    element_fth(c.clsH[3 * k], c.clsH[3 * k + 1], c.clsH[3 * k + 2], lay[p] ? st.V + 18 * (size_t)p : nullptr,
                lay[p] ? nullptr : st.s0 + 6 * (size_t)p, f33.data() + 33 * (size_t)k);
  }
  c.d_psetM.upload(M, c.stream);
  c.d_clsF33.upload(f33, c.stream);
  c.d_clsBorn.upload(clsBorn, c.stream);
  c.d_psetLayered.upload(lay, c.stream);
  if (st.D && st.s0) {
    c.d_stepD.upload(st.D, 36 * (size_t)c.npset, c.stream);
    c.d_stepS0.upload(st.s0, 6 * (size_t)c.npset, c.stream);
  } else {   // every set layered: no homogeneous data
    c.d_stepD.alloc(36 * (size_t)c.npset); c.d_stepD.zero(c.stream);
    c.d_stepS0.alloc(6 * (size_t)c.npset); c.d_stepS0.zero(c.stream);
  }
  c.stage = st.stage;
  c.stepReady = true;
  c.subReady = false;
}

void launch_class_condense(Context& c) {
  c.d_clsKc.alloc((size_t)c.ncls * 576);
  c.d_clsFc.alloc((size_t)c.ncls * 24);
  const int warps = 2;
  const size_t smem = (size_t)warps * 2048 * sizeof(double);
  TM_CUDA_CHECK(cudaFuncSetAttribute(k_class_condense, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  note_launch();
  k_class_condense<<<grid_for(c.ncls, warps), 32 * warps, smem, c.stream>>>(c.ncls, c.d_clsPset.p, c.d_clsH.p, c.d_psetM.p, c.d_clsF33.p,
                                                                          c.d_clsBorn.p, c.d_clsKc.p, c.d_clsFc.p);
  TM_CUDA_CHECK(cudaGetLastError());
}

void launch_assemble(Context& c) {
  const size_t tot = (size_t)NSLOT * c.nnp;
  c.d_val.alloc(tot * 9);
  c.d_rhs.alloc(3 * (size_t)c.nn);
  note_launch(2);
  {
  TimedLaunch tl(c, K_ASSEMBLE);
  k_assemble<<<grid_for(tot, 256), 256, 0, c.stream>>>(c.nn, c.nnp, c.nx, c.ny, c.nz, c.d_posNode.p, c.d_nodeIJK.p, c.d_nbr.p, c.d_cellElems.p,
                                                      c.d_eClass.p, c.d_eScale.p, c.d_eGroup.p, c.d_groupStage.p, c.stage, c.moduleStage ? 1 : 0,
                                                      c.d_clsKc.p, c.d_val.p);
  }
  TM_CUDA_CHECK(cudaGetLastError());
  k_assemble_rhs<<<grid_for(c.nn, 256), 256, 0, c.stream>>>(c.nn, c.nx, c.ny, c.nz, c.d_nodeIJK.p, c.d_cellElems.p, c.d_eClass.p,
                                                           c.d_eScale.p, c.d_eGroup.p, c.d_groupStage.p, c.stage, c.moduleStage ? 1 : 0,
                                                           c.d_clsBorn.p, c.d_clsFc.p, c.d_rhs.p);
  TM_CUDA_CHECK(cudaGetLastError());
}

void launch_constraints(Context& c) {
  c.d_isC.alloc(3 * (size_t)c.nn);
  c.d_isC.zero(c.stream);
  DBuf<int> d;
  d.upload(c.constr, c.stream);
  note_launch();
  if (!c.constr.empty())
    k_constraints<<<grid_for(c.constr.size(), 128), 128, 0, c.stream>>>(c.nnp, (int)c.constr.size(), d.p, c.d_pos.p, c.d_nbr.p,
                                                                       c.d_slotMask.p, c.d_val.p, c.d_rhs.p, c.d_isC.p);
  TM_CUDA_CHECK(cudaGetLastError());
  TM_CUDA_CHECK(cudaStreamSynchronize(c.stream));
  c.isC.assign(3 * (size_t)c.nn, 0);
  for (int d0 : c.constr) c.isC[d0] = 1;
}

void launch_scale(Context& c) {
  c.d_s.alloc(3 * (size_t)c.nn);
  note_launch(2);
  k_scale_diag<<<grid_for(c.nn, 256), 256, 0, c.stream>>>(c.nn, c.nnp, c.d_posNode.p, c.d_val.p, c.d_s.p);
  const size_t tot = (size_t)NSLOT * c.nn;
  k_scale_val<<<grid_for(tot, 256), 256, 0, c.stream>>>(c.nn, c.nnp, c.d_posNode.p, c.d_nbr.p, c.d_s.p, c.d_val.p);
  TM_CUDA_CHECK(cudaGetLastError());
}

void launch_scale_rhs(Context& c, const double* f, double* bs) {
  const size_t n = 3 * (size_t)c.nn;
  note_launch();
  k_mul<<<grid_for(n, 256), 256, 0, c.stream>>>(n, f, c.d_s.p, bs);
  TM_CUDA_CHECK(cudaGetLastError());
}

void launch_factor_columns(Context& c) {
  const int ncol = c.nx * c.ny;
  c.d_F.zero(c.stream);
  note_launch();
  k_factor_columns<<<grid_for(ncol, 128), 128, 0, c.stream>>>(ncol, c.nnp, c.d_colStart.p, c.d_pos.p, c.d_nbr.p, c.d_slotMask.p, c.d_val.p,
                                                             c.d_F.p, c.d_jitter.p);
  TM_CUDA_CHECK(cudaGetLastError());
}

void launch_w01(Context& c) {
  note_launch();
  k_w01<<<grid_for(c.nn, 256), 256, 0, c.stream>>>(c.nn, c.d_s.p, c.d_zp.p, c.d_W01.p);
  TM_CUDA_CHECK(cudaGetLastError());
}

void launch_factor_shell(Context& c, ShellLevel& L) {
  const int ncol = L.nx * L.ny;
  const int warps = 4;
  note_launch();
  k_factor_shell<<<grid_for(ncol, warps), 32 * warps, 0, c.stream>>>(ncol, L.d_colStart.p, L.d_rowPtr.p, L.d_col.p, L.d_val.p, L.d_cfPtr.p,
                                                                    L.d_cf.p, c.d_jitter.p);
  note_launch();
  k_shell_inverse<<<grid_for(ncol, warps), 32 * warps, 0, c.stream>>>(ncol, L.d_colStart.p, L.d_cfPtr.p, L.d_cf.p, L.d_cfInv.p);
  TM_CUDA_CHECK(cudaGetLastError());
}

// FP32 copies for the mixed-precision inner solve: operators, column factors and transfer weights
// (the coarsest level keeps its FP64 inverse)
void launch_to_fp32(Context& c) {
  auto conv = [&](const DBuf<double>& a, DBuf<float>& b) {
    b.alloc(a.n);
    if (a.n) { k_to_f32<<<grid_for(a.n, 256), 256, 0, c.stream>>>(a.n, a.p, b.p); note_launch(); }
  };
  if (!c.mf) launch_val_to_f32(c);   // the matrix-free level 0 reads no FP32 stencil
  conv(c.d_F, c.d_F32);
  conv(c.d_W01, c.d_W01_32);
  c.d_res0_32.alloc(3 * (size_t)c.nn);
  for (auto* r : {&c.d_r32, &c.d_z32, &c.d_p32, &c.d_q32, &c.d_d32}) r->alloc(3 * (size_t)c.nn);
  for (auto* L : c.shells) {
    if (L->coarsest) {
      L->d_b32.alloc(6 * (size_t)L->nn); L->d_x32.alloc(6 * (size_t)L->nn);
      continue;
    }
    conv(L->d_val, L->d_val32);
    conv(L->d_cfInv, L->d_cfInv32);
    conv(L->d_prolW, L->d_prolW32);
    L->d_b32.alloc(6 * (size_t)L->nn); L->d_x32.alloc(6 * (size_t)L->nn); L->d_res32.alloc(6 * (size_t)L->nn);
  }
  TM_CUDA_CHECK(cudaGetLastError());
}

void launch_accumulate_q(Context& c, const double* du, int nel, const int* elems, double* q) {
  if (nel <= 0) return;
  note_launch();
  k_accumulate_q<<<(nel + 3) / 4, 128, 0, c.stream>>>(nel, c.ne, elems, c.d_conn.p, c.d_eClass.p, c.d_clsPset.p, c.d_clsH.p, c.d_psetM.p,
                                                      c.d_clsF33.p, du, q);
  TM_CUDA_CHECK(cudaGetLastError());
}

void launch_element_strains_adjoint(Context& c, int np, const int* elem, const double* nat, const double* g, double* gq) {
  if (np <= 0) return;
  note_launch();
  k_element_strains_adjoint<<<grid_for(np, 128), 128, 0, c.stream>>>(np, c.ne, elem, c.d_eClass.p, c.d_clsH.p, nat, g, gq);
  TM_CUDA_CHECK(cudaGetLastError());
}

void launch_accumulate_q_adjoint(Context& c, int nel, const int* elems, const double* gq, double* gdu, double* gA) {
  if (nel <= 0) return;
  note_launch();
  k_accumulate_q_adjoint<<<(nel + 3) / 4, 128, 0, c.stream>>>(nel, c.ne, elems, c.d_eClass.p, c.d_clsPset.p, c.d_clsH.p, c.d_psetM.p,
                                                               c.d_clsF33.p, gq, gdu, gA);
  TM_CUDA_CHECK(cudaGetLastError());
}

void launch_element_strains(Context& c, int np, const int* elem, const double* q, const double* nat, double* eps) {
  if (np <= 0) return;
  note_launch();
  k_element_strains<<<grid_for(np, 128), 128, 0, c.stream>>>(np, c.ne, elem, c.d_eClass.p, c.d_clsH.p, q, nat, eps);
  TM_CUDA_CHECK(cudaGetLastError());
}

void launch_sample_plane(Context& c, const double* u, int k, int comp, int npts, const double* x, const double* y, double* out) {
  if (npts <= 0) return;
  if (!c.d_xs.p) {
    c.d_xs.upload(c.xs, c.stream);
    c.d_ys.upload(c.ys, c.stream);
    c.d_nodeId.upload(c.nodeId, c.stream);
  }
  note_launch();
  k_sample_plane<<<grid_for(npts, 128), 128, 0, c.stream>>>(npts, c.nx, c.ny, c.nz, c.d_xs.p, c.d_ys.p, c.d_nodeId.p, u, k, comp, x, y, out);
  TM_CUDA_CHECK(cudaGetLastError());
}

void launch_accumulate_state(Context& c, const double* du, int nel, const int* elems, int stride, double* state) {
  if (nel <= 0) return;
  note_launch();
  k_accumulate_state<<<(nel + 3) / 4, 128, 0, c.stream>>>(nel, c.ne, elems, c.d_conn.p, c.d_eClass.p, c.d_clsPset.p, c.d_clsH.p, c.d_psetM.p,
                                                          c.d_clsF33.p, c.d_clsBorn.p, c.d_psetLayered.p, c.d_stepD.p, c.d_stepS0.p,
                                                          c.d_subOff.p, c.d_subD.p, c.d_subS0.p, du, stride, state);
  TM_CUDA_CHECK(cudaGetLastError());
}

void launch_state_stress(Context& c, int np, const int* elem, const double* state, int stride, const double* nat, double* eps,
                         double* sig) {
  if (np <= 0) return;
  note_launch();
  k_state_stress<<<grid_for(np, 128), 128, 0, c.stream>>>(np, c.ne, elem, c.d_eClass.p, c.d_clsPset.p, c.d_clsH.p, c.d_eIJK.p, c.d_zs.p,
                                                         c.d_psetLayered.p, c.d_subOff.p, c.d_subZ.p, state, stride, nat, eps, sig);
  TM_CUDA_CHECK(cudaGetLastError());
}

namespace {
void sens_sums(Context& c, const double* u, const double* lam, const double* Kc, const double* Fc, double* outHost) {
  if (c.npset > SENS_MAXSET) fail(TM_BAD_INPUT, "sensitivities: too many property sets");
  DBuf<double> et, part;
  et.alloc(2 * (size_t)c.ne);
  const int chunk = 4096, nbk = (c.ne + chunk - 1) / chunk;
  part.alloc(2 * (size_t)nbk * c.npset);
  note_launch(2);
  k_sens_elements<<<(c.ne + 3) / 4, 128, 0, c.stream>>>(c.ne, c.d_conn.p, c.d_eClass.p, c.d_eScale.p, c.d_eGroup.p, c.d_groupStage.p, c.stage,
                                                       Kc, Fc, u, lam, et.p);
  k_sens_partial<<<nbk, 256, 0, c.stream>>>(c.ne, chunk, c.d_eClass.p, c.d_clsPset.p, c.npset, et.p, part.p);
  TM_CUDA_CHECK(cudaGetLastError());
  std::vector<double> h(2 * (size_t)nbk * c.npset);
  part.download(h.data(), h.size(), c.stream);
  TM_CUDA_CHECK(cudaStreamSynchronize(c.stream));
  for (int p = 0; p < 2 * c.npset; p++) outHost[p] = 0;
  for (int b = 0; b < nbk; b++)
    for (int p = 0; p < c.npset; p++) {
      outHost[2 * p] += h[2 * ((size_t)b * c.npset + p)];
      outHost[2 * p + 1] += h[2 * ((size_t)b * c.npset + p) + 1];
    }
}
}  // namespace

// directional sensitivities: per set a parameter t_m whose derivative of the set data (D, s0 or
// W, V) is dir; the shape matrices and element thermal loads are linear in those data, so their
// derivatives are the same maps applied to dir, and the condensation is differentiated exactly
// (k_class_dcondense); dJ/dt_m = lambda^T (df_m - dK_m u) summed over the set's elements. The base
// step's data are loaded again first (the class data of the step assembled last).
void sens_direction(Context& c, const tm_step& base, const tm_step& dir, const double* u, const double* lam, double* dJ) {
  const bool subWas = c.subReady;
  launch_shape_matrices(c, base);
  c.subReady = subWas;
  const int np = c.npset;
  std::vector<double> dMh((size_t)np * 6 * 1089), dF33((size_t)c.ncls * 33, 0.0);
  std::vector<double> zero108(108, 0.0), zero36(36, 0.0), zero18(18, 0.0), zero6(6, 0.0);
  for (int p = 0; p < np; p++) {
    const bool lay = base.psetLayered[p] != 0;
    const double* W = dir.W ? dir.W + 108 * (size_t)p : zero108.data();
    const double* D = dir.D ? dir.D + 36 * (size_t)p : zero36.data();
    shape_matrices(lay ? W : nullptr, lay ? nullptr : D, dMh.data() + (size_t)p * 6 * 1089);
  }
  for (int k = 0; k < c.ncls; k++) {
    const int p = c.clsPset[k];
    if (!base.psetBorn[p]) continue;
    const bool lay = base.psetLayered[p] != 0;
    const double* V = dir.V ? dir.V + 18 * (size_t)p : zero18.data();
    const double* S = dir.s0 ? dir.s0 + 6 * (size_t)p : zero6.data();
    element_fth(c.clsH[3 * k], c.clsH[3 * k + 1], c.clsH[3 * k + 2], lay ? V : nullptr, lay ? nullptr : S, dF33.data() + 33 * (size_t)k);
  }
  DBuf<double> dM, dF, dKc, dFc;
  dM.upload(dMh, c.stream);
  dF.upload(dF33, c.stream);
  dKc.alloc((size_t)c.ncls * 576);
  dFc.alloc((size_t)c.ncls * 24);
  const int warps = 2;
  const size_t smem = (size_t)warps * 2560 * sizeof(double);
  TM_CUDA_CHECK(cudaFuncSetAttribute(k_class_dcondense, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  note_launch();
  k_class_dcondense<<<grid_for(c.ncls, warps), 32 * warps, smem, c.stream>>>(c.ncls, c.d_clsPset.p, c.d_clsH.p, c.d_psetM.p, dM.p,
                                                                            c.d_clsF33.p, dF.p, c.d_clsBorn.p, dKc.p, dFc.p);
  TM_CUDA_CHECK(cudaGetLastError());
  std::vector<double> sums(2 * (size_t)np);
  sens_sums(c, u, lam, dKc.p, dFc.p, sums.data());
  for (int p = 0; p < np; p++) dJ[p] = sums[2 * p + 1] - sums[2 * p];
  TM_CUDA_CHECK(cudaStreamSynchronize(c.stream));
}

// the element terms of the warpage sensitivities summed per property set: out[2p] = sum over the
// set's elements of s_e lambda^T K_e u, out[2p+1] = sum of s_e lambda^T f_e
void launch_sens(Context& c, const double* u, const double* lam, double* outHost) {
  sens_sums(c, u, lam, c.d_clsKc.p, c.d_clsFc.p, outHost);
}

}  // namespace tmg
