// CPU FP64 oracle of the reference solve path -- TEST INFRASTRUCTURE ONLY.
//
// This file restates, in plain C++, the algorithms of the reference tool
// (ProtonNeutronElectron69/Packaging-TM-modeling-tool, JavaScript) that the
// GPU library replaces. It is the checker for the parity tests and the timed
// CPU baseline of bench.py; nothing in the product links or calls it.
//
// Parity is pinned by the reference's own analytic known-answer tests
// (src/core/15-verify.js V1, V2, V3, V4, V6, V16, V18(4)), re-implemented in
// tests/test_oracle_known_answers.py, and by its published whole-package
// results on its own models (V5, V8, V9, V11, V18, the default package's room-
// temperature warpage), reproduced through the host's restated model building
// in tests/test_host_analysis.py, tests/test_host_thermal.py and
// tests/test_host_modules.py (V18's series column of one point there); the reference
// publishes no golden vector files and its JavaScript cannot be run here (no
// JS engine).
//
// Loop orders follow the reference line by line so that the summation order
// of every dot product, matvec and factorisation is the same; the file is
// compiled with -ffp-contract=off because JavaScript has no fused multiply-add.
//
// Sections and the reference lines they follow:
//   mesher          src/core/06-mesher.js:14-72, 74-84, 112-116
//   element         src/core/07-element.js:12-121
//   dense algebra   src/core/01-util.js:70-142, 176-190
//   assembly        src/core/08-sparse.js:7-43, src/core/09-assembly.js:23-165, 318-332, 392-464
//   solver          src/core/10-solver.js:1-1043
//   recovery, post  src/core/09-assembly.js:480-533, 07-element.js:127-142, 12-post.js:30-109
//   Anand           src/core/13-fatigue.js:13-293, 379-455
#include <cmath>
#include <cstdint>
#include <cstring>
#include <algorithm>
#include <array>
#include <cstdio>
#include <chrono>
#include <map>
#include <memory>
#include <set>
#include <stdexcept>
#include <string>
#include <vector>

namespace {

using std::vector;
typedef vector<double> dvec;
typedef vector<int> ivec;

double now_ms() {
  using namespace std::chrono;
  return duration<double, std::milli>(steady_clock::now().time_since_epoch()).count();
}

// ---- constants (src/core/00-constants.js) ------------------------------------
const double UNBORN_SCALE = 1e-6;          // :18
const double PCG_TOL = 1e-8;               // :60
const int PCG_MAXIT = 2000;                // :61
const int WARM_START_MAX = 20;             // :62
const double REBUILD_FACTOR = 2;           // :63
const int REBUILD_MIN_ITERS = 30;          // :64
const int MG_COARSEST_COLS = 9;            // :79
const int MG_COARSEST_DOF = 900;           // :80
const double MG_MIN_COARSENING = 0.7;      // :81
const double CHOL_JITTER = 1e-12;          // :82
const double IC_SHIFT0 = 1e-3;             // :83
const double IC_SHIFT_MAX = 1;             // :84
const int COLUMN_NEWTON_MAXIT = 20;        // :121
const double COLUMN_STRESS_TOL = 1e-3;     // :122
const int ANAND_NEWTON_MAXIT = 60;         // :123
const double ANAND_TOL = 1e-11;            // :124
const double KELVIN = 273.15;              // :15
const int TGRID_MIN = -80, TGRID_MAX = 300; // :12-13
const int TGRID_N = TGRID_MAX - TGRID_MIN + 1;

// compliant parts that split a column into separate shell aggregates (10-solver.js:248)
// PART ids: 06-mesher.js:3-4 (SOLDER 1, UF_BUMP 2, UF_FILLET 3, TIM 5, LIDADH 7, STIFFADH 9)
bool is_compliant_part(int p) { return p == 1 || p == 2 || p == 3 || p == 5 || p == 7 || p == 9; }

// ---- dense algebra (src/core/01-util.js) ---------------------------------------
// cholDense :70-91
int cholDense(double* A, int n, double rel) {
  double dmax = 0;
  for (int i = 0; i < n; i++) dmax = std::max(dmax, std::fabs(A[i * n + i]));
  const double jitter = (rel != 0 ? rel : CHOL_JITTER) * (dmax != 0 ? dmax : 1);
  int fixes = 0;
  for (int j = 0; j < n; j++) {
    const int rj = j * n;
    double d = A[rj + j];
    for (int k = 0; k < j; k++) d -= A[rj + k] * A[rj + k];
    if (!(d > jitter)) { d = std::max(std::fabs(d), jitter); fixes++; }
    const double ljj = std::sqrt(d);
    A[rj + j] = ljj;
    const double inv = 1 / ljj;
    for (int i = j + 1; i < n; i++) {
      const int ri = i * n;
      double s = A[ri + j];
      for (int k = 0; k < j; k++) s -= A[ri + k] * A[rj + k];
      A[ri + j] = s * inv;
    }
  }
  return fixes;
}

// cholSolveDense :94-107 (and cholSolveDenseOff, 10-solver.js:497-509)
void cholSolveDenseOff(const double* L, int n, double* b) {
  for (int i = 0; i < n; i++) {
    double s = b[i];
    const int ri = i * n;
    for (int k = 0; k < i; k++) s -= L[ri + k] * b[k];
    b[i] = s / L[ri + i];
  }
  for (int i = n - 1; i >= 0; i--) {
    double s = b[i];
    for (int k = i + 1; k < n; k++) s -= L[k * n + i] * b[k];
    b[i] = s / L[i * n + i];
  }
}

// invDense :110-134 (Gauss-Jordan with partial pivoting); returns false when singular
bool invDense(const double* A, int n, double* R) {
  const int w = 2 * n;
  dvec M((size_t)n * w, 0.0);
  for (int i = 0; i < n; i++) {
    for (int j = 0; j < n; j++) M[i * w + j] = A[i * n + j];
    M[i * w + n + i] = 1;
  }
  for (int c = 0; c < n; c++) {
    int p = c; double best = std::fabs(M[c * w + c]);
    for (int r = c + 1; r < n; r++) { double v = std::fabs(M[r * w + c]); if (v > best) { best = v; p = r; } }
    if (best == 0) return false;
    if (p != c) for (int j = 0; j < w; j++) std::swap(M[c * w + j], M[p * w + j]);
    const double inv = 1 / M[c * w + c];
    for (int j = 0; j < w; j++) M[c * w + j] *= inv;
    for (int r = 0; r < n; r++) {
      if (r == c) continue;
      const double f = M[r * w + c];
      if (f == 0) continue;
      for (int j = 0; j < w; j++) M[r * w + j] -= f * M[c * w + j];
    }
  }
  for (int i = 0; i < n; i++) for (int j = 0; j < n; j++) R[i * n + j] = M[i * w + n + j];
  return true;
}

// solveDense :137-142
bool solveDense(const double* A, int n, const double* b, double* x) {
  dvec Ai((size_t)n * n);
  if (!invDense(A, n, Ai.data())) return false;
  for (int i = 0; i < n; i++) { double s = 0; for (int j = 0; j < n; j++) s += Ai[i * n + j] * b[j]; x[i] = s; }
  return true;
}

// inv3 (07-element.js:146-153)
double inv3(const double* J, double* out) {
  const double a = J[0], b = J[1], c = J[2], d = J[3], e = J[4], f = J[5], g = J[6], h = J[7], i = J[8];
  const double det = a * (e * i - f * h) - b * (d * i - f * g) + c * (d * h - e * g);
  out[0] = (e * i - f * h) / det; out[1] = (c * h - b * i) / det; out[2] = (b * f - c * e) / det;
  out[3] = (f * g - d * i) / det; out[4] = (a * i - c * g) / det; out[5] = (c * d - a * f) / det;
  out[6] = (d * h - e * g) / det; out[7] = (b * g - a * h) / det; out[8] = (a * e - b * d) / det;
  return det;
}

double dot(const dvec& a, const dvec& b) { double s = 0; for (size_t i = 0; i < a.size(); i++) s += a[i] * b[i]; return s; }
double norm2(const dvec& a) { return std::sqrt(dot(a, a)); }
void axpy(double alpha, const dvec& x, dvec& y) { for (size_t i = 0; i < y.size(); i++) y[i] += alpha * x[i]; }

// ---- element (src/core/07-element.js, 09-assembly.js:23-133) ---------------------
const int HEX_XI[8] = {-1, 1, 1, -1, -1, 1, 1, -1};
const int HEX_ETA[8] = {-1, -1, 1, 1, -1, -1, 1, 1};
const int HEX_ZETA[8] = {-1, -1, -1, -1, 1, 1, 1, 1};
const int NFUN = 11;
const int VOIGT_IDX[3][3] = {{0, 3, 5}, {3, 1, 4}, {5, 4, 2}};

struct Univ { double G[3 * 9 * 121]; double g[3 * 3 * 11]; double GH[9 * 121]; double gH[3 * 11]; };

// UNIV (09-assembly.js:26-60)
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
      for (int r = 0; r < 3; r++) {
        for (int a = 0; a < 11; a++) {
          U.g[(j * 3 + r) * 11 + a] += d[r][a];
          U.gH[r * 11 + a] += simpson[j] * d[r][a];
          for (int s = 0; s < 3; s++) for (int b = 0; b < 11; b++) {
            const double v = d[r][a] * d[s][b];
            U.G[((j * 9 + r * 3 + s) * 121) + a * 11 + b] += v;
            U.GH[(r * 3 + s) * 121 + a * 11 + b] += simpson[j] * v;
          }
        }
      }
    }
  }
  done = true;
  return U;
}

// shapeMatrices (09-assembly.js:69-93); Wst (108) for a layered section or D (36)
void shapeMatrices(const double* Wst, const double* D, double* M) {
  const Univ& U = univ();
  std::fill(M, M + 6 * 1089, 0.0);
  const int nst = D ? 1 : 3;
  const int PAIR[6][3] = {{0, 0, 0}, {1, 1, 1}, {2, 2, 2}, {3, 0, 1}, {4, 1, 2}, {5, 2, 0}};
  for (int j = 0; j < nst; j++) {
    const double* Wj = D ? D : Wst + 36 * j;
    for (int pi = 0; pi < 6; pi++) {
      const int m = PAIR[pi][0], r = PAIR[pi][1], s = PAIR[pi][2];
      double* Mm = M + m * 1089;
      int rsList[2][2] = {{r, s}, {s, r}};
      const int nrs = r == s ? 1 : 2;
      for (int t = 0; t < nrs; t++) {
        const int rr = rsList[t][0], ss = rsList[t][1];
        const double* Gb = D ? U.GH + (rr * 3 + ss) * 121 : U.G + (j * 9 + rr * 3 + ss) * 121;
        for (int p = 0; p < 3; p++) for (int q = 0; q < 3; q++) {
          const double dv = Wj[VOIGT_IDX[p][rr] * 6 + VOIGT_IDX[q][ss]];
          if (dv == 0) continue;
          for (int a = 0; a < NFUN; a++) {
            const int row = (3 * a + p) * 33 + q, ga = a * 11;
            for (int b = 0; b < NFUN; b++) Mm[row + 3 * b] += dv * Gb[ga + b];
          }
        }
      }
    }
  }
}

// elementK33Fast (09-assembly.js:96-108)
void elementK33Fast(double hx, double hy, double hz, const double* M, double* K) {
  const double V8 = hx * hy * hz / 8;
  const double c[6] = {V8 * 4 / (hx * hx), V8 * 4 / (hy * hy), V8 * 4 / (hz * hz), V8 * 4 / (hx * hy), V8 * 4 / (hy * hz), V8 * 4 / (hz * hx)};
  for (int i = 0; i < 33; i++) {
    const int ri = i * 33;
    for (int j = i; j < 33; j++) {
      const int o = ri + j;
      K[o] = c[0] * M[o] + c[1] * M[1089 + o] + c[2] * M[2178 + o] + c[3] * M[3267 + o] + c[4] * M[4356 + o] + c[5] * M[5445 + o];
    }
  }
  for (int i = 0; i < 33; i++) for (int j = i + 1; j < 33; j++) K[j * 33 + i] = K[i * 33 + j];
}

// elementFth (09-assembly.js:115-133); Sst (18) for a layered section or s0 (6)
void elementFth(double hx, double hy, double hz, const double* Sst, const double* s0, double* f) {
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
        const double sv = c * Sj[VOIGT_IDX[p][r]];
        if (sv == 0) continue;
        for (int a = 0; a < NFUN; a++) f[3 * a + p] += sv * gb[a];
      }
    }
  }
}

// condense33 (07-element.js:88-121)
void condense33(const double* K, const double* f, double* Kc, double* fc, double* Xout) {
  double Kaa[81], col[9], X[216], xf[9];
  for (int i = 0; i < 9; i++) for (int j = 0; j < 9; j++) Kaa[i * 9 + j] = K[(24 + i) * 33 + 24 + j];
  cholDense(Kaa, 9, 1e-14);
  for (int j = 0; j < 24; j++) {
    for (int i = 0; i < 9; i++) col[i] = K[(24 + i) * 33 + j];
    cholSolveDenseOff(Kaa, 9, col);
    for (int i = 0; i < 9; i++) X[i * 24 + j] = col[i];
  }
  for (int i = 0; i < 24; i++) {
    for (int j = 0; j < 24; j++) {
      double s = K[i * 33 + j];
      for (int q = 0; q < 9; q++) s -= K[i * 33 + 24 + q] * X[q * 24 + j];
      Kc[i * 24 + j] = s;
    }
  }
  for (int i = 0; i < 24; i++) for (int j = i + 1; j < 24; j++) { const double v = 0.5 * (Kc[i * 24 + j] + Kc[j * 24 + i]); Kc[i * 24 + j] = Kc[j * 24 + i] = v; }
  if (f) {
    for (int i = 0; i < 9; i++) col[i] = f[24 + i];
    cholSolveDenseOff(Kaa, 9, col);
    for (int i = 0; i < 9; i++) xf[i] = col[i];
    for (int i = 0; i < 24; i++) {
      double s = f[i];
      for (int q = 0; q < 9; q++) s -= K[i * 33 + 24 + q] * xf[q];
      fc[i] = s;
    }
  }
  if (Xout) std::memcpy(Xout, X, sizeof(X));
}

// boxDerivs (07-element.js:19-30)
void boxDerivs(double hx, double hy, double hz, double xi, double eta, double zeta, double* dx, double* dy, double* dz) {
  const double sx = 2 / hx, sy = 2 / hy, sz = 2 / hz;
  for (int a = 0; a < 8; a++) {
    const double xa = HEX_XI[a], ya = HEX_ETA[a], za = HEX_ZETA[a];
    dx[a] = xa * (1 + ya * eta) * (1 + za * zeta) * 0.125 * sx;
    dy[a] = ya * (1 + xa * xi) * (1 + za * zeta) * 0.125 * sy;
    dz[a] = za * (1 + xa * xi) * (1 + ya * eta) * 0.125 * sz;
  }
  dx[8] = -2 * xi * sx; dy[8] = 0; dz[8] = 0;
  dx[9] = 0; dy[9] = -2 * eta * sy; dz[9] = 0;
  dx[10] = 0; dy[10] = 0; dz[10] = -2 * zeta * sz;
}

// accumulatePoint (07-element.js:42-75)
void accumulatePoint(const double* dx, const double* dy, const double* dz, const double* D, const double* s0, double w, double* K, double* f) {
  double DB[NFUN * 18];
  for (int b = 0; b < NFUN; b++) {
    const double bx = dx[b], by = dy[b], bz = dz[b];
    const int o = b * 18;
    for (int r = 0; r < 6; r++) {
      const int d = r * 6;
      DB[o + r * 3] = D[d] * bx + D[d + 3] * by + D[d + 5] * bz;
      DB[o + r * 3 + 1] = D[d + 1] * by + D[d + 3] * bx + D[d + 4] * bz;
      DB[o + r * 3 + 2] = D[d + 2] * bz + D[d + 4] * by + D[d + 5] * bx;
    }
  }
  for (int a = 0; a < NFUN; a++) {
    const double ax = dx[a] * w, ay = dy[a] * w, az = dz[a] * w;
    if (ax == 0 && ay == 0 && az == 0) continue;
    const int ra = 3 * a;
    for (int b = a; b < NFUN; b++) {
      const int o = b * 18;
      for (int c = 0; c < 3; c++) {
        const double k0 = ax * DB[o + c] + ay * DB[o + 9 + c] + az * DB[o + 15 + c];
        const double k1 = ay * DB[o + 3 + c] + ax * DB[o + 9 + c] + az * DB[o + 12 + c];
        const double k2 = az * DB[o + 6 + c] + ay * DB[o + 12 + c] + ax * DB[o + 15 + c];
        K[ra * 33 + 3 * b + c] += k0;
        K[(ra + 1) * 33 + 3 * b + c] += k1;
        K[(ra + 2) * 33 + 3 * b + c] += k2;
      }
    }
    if (s0) {
      f[ra] += ax * s0[0] + ay * s0[3] + az * s0[5];
      f[ra + 1] += ay * s0[1] + ax * s0[3] + az * s0[4];
      f[ra + 2] += az * s0[2] + ay * s0[4] + ax * s0[5];
    }
  }
}

void symmetrize33(double* K) {
  for (int a = 0; a < NFUN; a++) for (int b = a + 1; b < NFUN; b++)
    for (int p = 0; p < 3; p++) for (int q = 0; q < 3; q++) K[(3 * b + q) * 33 + 3 * a + p] = K[(3 * a + p) * 33 + 3 * b + q];
}

// general (distorted) hexahedron with 2x2x2 Gauss (07-element.js:156-205), for the patch test
double generalDerivs(const double* X, double xi, double eta, double zeta, const double* J0inv, double detJ0, double* dx, double* dy, double* dz) {
  double dNxi[8], dNeta[8], dNzeta[8];
  for (int a = 0; a < 8; a++) {
    const double xa = HEX_XI[a], ya = HEX_ETA[a], za = HEX_ZETA[a];
    dNxi[a] = xa * (1 + ya * eta) * (1 + za * zeta) * 0.125;
    dNeta[a] = ya * (1 + xa * xi) * (1 + za * zeta) * 0.125;
    dNzeta[a] = za * (1 + xa * xi) * (1 + ya * eta) * 0.125;
  }
  double J[9] = {0}, Ji[9];
  for (int a = 0; a < 8; a++) for (int j = 0; j < 3; j++) {
    J[j] += dNxi[a] * X[3 * a + j]; J[3 + j] += dNeta[a] * X[3 * a + j]; J[6 + j] += dNzeta[a] * X[3 * a + j];
  }
  const double detJ = inv3(J, Ji);
  for (int a = 0; a < 8; a++) {
    dx[a] = Ji[0] * dNxi[a] + Ji[1] * dNeta[a] + Ji[2] * dNzeta[a];
    dy[a] = Ji[3] * dNxi[a] + Ji[4] * dNeta[a] + Ji[5] * dNzeta[a];
    dz[a] = Ji[6] * dNxi[a] + Ji[7] * dNeta[a] + Ji[8] * dNzeta[a];
  }
  const double r = detJ0 / detJ;
  const double gp[3][3] = {{-2 * xi, 0, 0}, {0, -2 * eta, 0}, {0, 0, -2 * zeta}};
  for (int m = 0; m < 3; m++) {
    const double* g = gp[m];
    dx[8 + m] = r * (J0inv[0] * g[0] + J0inv[1] * g[1] + J0inv[2] * g[2]);
    dy[8 + m] = r * (J0inv[3] * g[0] + J0inv[4] * g[1] + J0inv[5] * g[2]);
    dz[8 + m] = r * (J0inv[6] * g[0] + J0inv[7] * g[1] + J0inv[8] * g[2]);
  }
  return detJ;
}

void generalElement(const double* X, const double* D, double* Kc, double* Xcond) {
  double K[1089] = {0}, f[33] = {0}, dx[NFUN], dy[NFUN], dz[NFUN];
  double J[9] = {0}, J0i[9];
  for (int a = 0; a < 8; a++) for (int j = 0; j < 3; j++) {
    J[j] += HEX_XI[a] * 0.125 * X[3 * a + j]; J[3 + j] += HEX_ETA[a] * 0.125 * X[3 * a + j]; J[6 + j] += HEX_ZETA[a] * 0.125 * X[3 * a + j];
  }
  const double det0 = inv3(J, J0i);
  const double GP2 = 1 / std::sqrt(3.0);
  for (int a = 0; a < 2; a++) for (int b = 0; b < 2; b++) for (int c = 0; c < 2; c++) {
    const double detJ = generalDerivs(X, a ? GP2 : -GP2, b ? GP2 : -GP2, c ? GP2 : -GP2, J0i, det0, dx, dy, dz);
    accumulatePoint(dx, dy, dz, D, nullptr, detJ, K, f);
  }
  symmetrize33(K);
  double fc[24];
  condense33(K, nullptr, Kc, fc, Xcond);
}

// ---- mesh (src/core/06-mesher.js:14-72) ---------------------------------------
struct Mesh {
  int nx, ny, nz;
  dvec xs, ys, zs;
  int nn = 0, ne = 0;
  dvec coords;
  ivec nodeId, conn, eIJK, colStart, cellElems, eGroup, ePart;
  dvec eScale;
  ivec featureX, featureY;
  bool hasFeatures = false;
};

// cellGroup/cellPart/cellScale hold up to two phases per cell (group < 0: none)
void buildStructuredMesh(Mesh& m, const int* cellGroup, const int* cellPart, const double* cellScale) {
  const int nx = m.nx, ny = m.ny, nz = m.nz, ncy = ny - 1, ncz = nz - 1;
  const int ncells = (nx - 1) * ncy * ncz;
  m.cellElems.assign((size_t)ncells * 2, -1);
  std::vector<uint8_t> exist((size_t)nx * ny * nz, 0);
  ivec eCell;
  for (int i = 0; i < nx - 1; i++) for (int j = 0; j < ncy; j++) for (int k = 0; k < ncz; k++) {
    const int c = (i * ncy + j) * ncz + k;
    int cnt = 0;
    for (int q = 0; q < 2; q++) {
      if (cellGroup[2 * c + q] < 0) continue;
      m.cellElems[c * 2 + cnt] = (int)m.eGroup.size();
      m.eGroup.push_back(cellGroup[2 * c + q]); m.ePart.push_back(cellPart[2 * c + q]); m.eScale.push_back(cellScale[2 * c + q]); eCell.push_back(c);
      cnt++;
    }
    if (!cnt) continue;
    for (int di = 0; di < 2; di++) for (int dj = 0; dj < 2; dj++) for (int dk = 0; dk < 2; dk++) exist[((size_t)(i + di) * ny + j + dj) * nz + k + dk] = 1;
  }
  m.nodeId.assign((size_t)nx * ny * nz, -1);
  int nn = 0;
  for (size_t q = 0; q < exist.size(); q++) if (exist[q]) m.nodeId[q] = nn++;
  m.nn = nn;
  m.coords.assign((size_t)nn * 3, 0.0);
  for (int i = 0; i < nx; i++) for (int j = 0; j < ny; j++) for (int k = 0; k < nz; k++) {
    const int id = m.nodeId[((size_t)i * ny + j) * nz + k];
    if (id < 0) continue;
    m.coords[3 * id] = m.xs[i]; m.coords[3 * id + 1] = m.ys[j]; m.coords[3 * id + 2] = m.zs[k];
  }
  const int ne = (int)m.eGroup.size();
  m.ne = ne;
  m.conn.assign((size_t)ne * 8, 0);
  m.eIJK.assign((size_t)ne * 3, 0);
  const int loc[8][3] = {{0, 0, 0}, {1, 0, 0}, {1, 1, 0}, {0, 1, 0}, {0, 0, 1}, {1, 0, 1}, {1, 1, 1}, {0, 1, 1}};
  for (int e = 0; e < ne; e++) {
    const int c = eCell[e];
    const int k = c % ncz, j = (c / ncz) % ncy, i = c / (ncz * ncy);
    m.eIJK[3 * e] = i; m.eIJK[3 * e + 1] = j; m.eIJK[3 * e + 2] = k;
    for (int a = 0; a < 8; a++) m.conn[8 * e + a] = m.nodeId[((size_t)(i + loc[a][0]) * ny + j + loc[a][1]) * nz + k + loc[a][2]];
  }
  m.colStart.assign((size_t)nx * ny + 1, 0);
  int cnt = 0;
  for (int c = 0; c < nx * ny; c++) {
    m.colStart[c] = cnt;
    for (int k = 0; k < nz; k++) if (m.nodeId[(size_t)c * nz + k] >= 0) cnt++;
  }
  m.colStart[nx * ny] = cnt;
}

// nearestNodeOnPlane (06-mesher.js:75-84)
int nearestNodeOnPlane(const Mesh& m, double x, double y, int k) {
  int best = -1; double bd = INFINITY;
  for (int i = 0; i < m.nx; i++) for (int j = 0; j < m.ny; j++) {
    const int id = m.nodeId[((size_t)i * m.ny + j) * m.nz + k];
    if (id < 0) continue;
    const double d = std::hypot(m.xs[i] - x, m.ys[j] - y);
    if (d < bd - 1e-12) { bd = d; best = id; }
  }
  return best;
}

// constraints321 (06-mesher.js:112-116)
ivec constraints321(const Mesh& m, double a) {
  const int n0 = nearestNodeOnPlane(m, 0, 0, 0), n1 = nearestNodeOnPlane(m, a, 0, 0), n2 = nearestNodeOnPlane(m, 0, a, 0);
  return ivec{3 * n0, 3 * n0 + 1, 3 * n0 + 2, 3 * n1 + 1, 3 * n1 + 2, 3 * n2 + 2};
}

// ---- block CSR (src/core/08-sparse.js:7-39, 09-assembly.js:136-165) ------------------
struct Pattern { int n = 0; ivec rowPtr, col, diag; int nb = 0; };

Pattern bcsrFromElements(int nn, const ivec& conn, int ne, int npe) {
  ivec cnt(nn + 1, 0);
  for (int q = 0; q < ne * npe; q++) cnt[conn[q] + 1]++;
  for (int i = 0; i < nn; i++) cnt[i + 1] += cnt[i];
  ivec adj((size_t)ne * npe), fill(cnt.begin(), cnt.begin() + nn);
  for (int e = 0; e < ne; e++) for (int a = 0; a < npe; a++) { const int n = conn[e * npe + a]; adj[fill[n]++] = e; }
  ivec mark(nn, -1);
  Pattern P; P.n = nn; P.rowPtr.assign(nn + 1, 0);
  for (int i = 0; i < nn; i++) {
    int c = 0;
    for (int q = cnt[i]; q < cnt[i + 1]; q++) {
      const int e = adj[q];
      for (int a = 0; a < npe; a++) { const int j = conn[e * npe + a]; if (j >= i && mark[j] != i) { mark[j] = i; c++; } }
    }
    P.rowPtr[i + 1] = P.rowPtr[i] + c;
  }
  P.col.assign(P.rowPtr[nn], 0);
  std::fill(mark.begin(), mark.end(), -1);
  ivec tmp;
  for (int i = 0; i < nn; i++) {
    tmp.clear();
    for (int q = cnt[i]; q < cnt[i + 1]; q++) {
      const int e = adj[q];
      for (int a = 0; a < npe; a++) { const int j = conn[e * npe + a]; if (j >= i && mark[j] != i) { mark[j] = i; tmp.push_back(j); } }
    }
    std::sort(tmp.begin(), tmp.end());
    std::copy(tmp.begin(), tmp.end(), P.col.begin() + P.rowPtr[i]);
  }
  P.nb = P.rowPtr[nn];
  return P;
}

Pattern fullPatternFromUpper(const Pattern& U) {
  const int n = U.n;
  ivec cnt(n + 1, 0);
  for (int i = 0; i < n; i++) for (int k = U.rowPtr[i]; k < U.rowPtr[i + 1]; k++) { const int j = U.col[k]; cnt[i + 1]++; if (j != i) cnt[j + 1]++; }
  for (int i = 0; i < n; i++) cnt[i + 1] += cnt[i];
  Pattern P; P.n = n; P.rowPtr = cnt; P.col.assign(cnt[n], 0);
  ivec fill(cnt.begin(), cnt.begin() + n);
  for (int i = 0; i < n; i++) for (int k = U.rowPtr[i]; k < U.rowPtr[i + 1]; k++) { const int j = U.col[k]; P.col[fill[i]++] = j; if (j != i) P.col[fill[j]++] = i; }
  for (int i = 0; i < n; i++) std::sort(P.col.begin() + cnt[i], P.col.begin() + cnt[i + 1]);
  P.diag.assign(n, 0);
  for (int i = 0; i < n; i++) for (int k = cnt[i]; k < cnt[i + 1]; k++) if (P.col[k] == i) { P.diag[i] = k; break; }
  P.nb = cnt[n];
  return P;
}

// fullMatVec (09-assembly.js:151-165)
void fullMatVec(const Pattern& P, const double* val, const double* x, double* y) {
  const int n = P.n;
  for (int i = 0; i < n; i++) {
    double y0 = 0, y1 = 0, y2 = 0;
    for (int k = P.rowPtr[i]; k < P.rowPtr[i + 1]; k++) {
      const int j = P.col[k]; const size_t v = 9 * (size_t)k;
      const double xj0 = x[3 * j], xj1 = x[3 * j + 1], xj2 = x[3 * j + 2];
      y0 += val[v] * xj0 + val[v + 1] * xj1 + val[v + 2] * xj2;
      y1 += val[v + 3] * xj0 + val[v + 4] * xj1 + val[v + 5] * xj2;
      y2 += val[v + 6] * xj0 + val[v + 7] * xj1 + val[v + 8] * xj2;
    }
    y[3 * i] = y0; y[3 * i + 1] = y1; y[3 * i + 2] = y2;
  }
}

// blockMatVec (10-solver.js:134-153)
void blockMatVec(const Pattern& P, const double* val, int b, const double* x, double* y) {
  if (b == 3) { fullMatVec(P, val, x, y); return; }
  const int n = P.n;
  for (int i = 0; i < n; i++) {
    double yy[6] = {0, 0, 0, 0, 0, 0};
    for (int k = P.rowPtr[i]; k < P.rowPtr[i + 1]; k++) {
      const int j = P.col[k]; const size_t v = 36 * (size_t)k; const int o = 6 * j;
      for (int r = 0; r < 6; r++) {
        const double* vr = val + v + 6 * r;
        yy[r] += vr[0] * x[o] + vr[1] * x[o + 1] + vr[2] * x[o + 2] + vr[3] * x[o + 3] + vr[4] * x[o + 4] + vr[5] * x[o + 5];
      }
    }
    for (int r = 0; r < 6; r++) y[6 * i + r] = yy[r];
  }
}

int findBlock(const Pattern& P, int row, int colj) {
  int lo = P.rowPtr[row], hi = P.rowPtr[row + 1] - 1;
  while (lo <= hi) { const int mid = (lo + hi) >> 1; const int v = P.col[mid]; if (v == colj) return mid; if (v < colj) lo = mid + 1; else hi = mid - 1; }
  return -1;
}

// ---- FE model: assembly with element birth and constraints (09-assembly.js:208-464) -----
// A property set is a homogeneous group (D 36, s0 6) or a layered section (W 108, V 18).
struct PropSet {
  bool layered = false; double D[36]; double s0[6]; double W[108]; double V[18]; bool born = true; double M[6 * 1089];
  // layered sets: per sub-layer its z range, step-mean stiffness and thermal stress increment
  // (sectionSubMeanD / sectionSubStress, 04-homogenize.js:196-204), for the stress histories
  int nsub = 0; dvec subZ, subD, subS0;
};

struct Model {
  Mesh mesh;
  Pattern upper, pattern;
  ivec bmap;
  dvec val;
  int ndof = 0;
  ivec constraints;
  std::vector<uint8_t> isConstrained;
  ivec ePset;             // property set of every element
  ivec groupStage;        // birth stage per group
  std::vector<PropSet> psets;
  int stage = 0;
  bool assembled = false;
  // stacked modules (09-assembly.js:227, 392-443): the package's then the modules' 3-2-1 supports,
  // and for a module stage assembled last its born elements and the nodes they touch
  ivec moduleConstraints;
  bool moduleStage = false;
  std::vector<uint8_t> actElem, actNode;
};

// moduleStageSet / moduleStageConstraints (09-assembly.js:427-440): the elements born in the stage,
// the nodes they touch, and the module constraints plus every DOF of the other nodes (sorted)
ivec moduleStageSet(Model& M, int stage) {
  const Mesh& m = M.mesh;
  M.actElem.assign(m.ne, 0);
  M.actNode.assign(m.nn, 0);
  for (int e = 0; e < m.ne; e++) {
    if (M.groupStage[m.eGroup[e]] > stage) continue;
    M.actElem[e] = 1;
    for (int a = 0; a < 8; a++) M.actNode[m.conn[8 * e + a]] = 1;
  }
  std::vector<uint8_t> fixed(M.ndof, 0);
  for (int d : M.moduleConstraints) fixed[d] = 1;
  for (int n = 0; n < m.nn; n++) if (!M.actNode[n]) fixed[3 * n] = fixed[3 * n + 1] = fixed[3 * n + 2] = 1;
  ivec dofs;
  for (int d = 0; d < M.ndof; d++) if (fixed[d]) dofs.push_back(d);
  return dofs;
}

void blockMap(Model& M) {
  const Mesh& m = M.mesh; const Pattern& P = M.pattern;
  M.bmap.assign((size_t)m.ne * 64, -1);
  for (int e = 0; e < m.ne; e++) for (int a = 0; a < 8; a++) {
    const int na = m.conn[8 * e + a];
    for (int b = 0; b < 8; b++) M.bmap[((size_t)e * 8 + a) * 8 + b] = findBlock(P, na, m.conn[8 * e + b]);
  }
}

// applyConstraints (09-assembly.js:445-464)
void applyConstraints(Model& M, double* rhs, const ivec& dofs) {
  const Pattern& P = M.pattern; double* val = M.val.data();
  M.isConstrained.assign(M.ndof, 0);
  for (int d : dofs) M.isConstrained[d] = 1;
  for (int d : dofs) {
    const int i = d / 3, p = d % 3;
    for (int k = P.rowPtr[i]; k < P.rowPtr[i + 1]; k++) {
      const int j = P.col[k]; const size_t v = 9 * (size_t)k;
      for (int q = 0; q < 3; q++) { if (3 * j + q != d) val[v + 3 * p + q] = 0; else if (val[v + 3 * p + q] == 0) val[v + 3 * p + q] = 1; }
      const int kk = findBlock(P, j, i);
      const size_t w = 9 * (size_t)kk;
      for (int q = 0; q < 3; q++) { if (3 * j + q != d) val[w + 3 * q + p] = 0; }
    }
    if (rhs) rhs[d] = 0;
  }
}

// assembleStep (09-assembly.js:392-424) with prepareStep's shape matrices (:346-365)
void assembleStep(Model& M, double* rhs, bool noConstraints) {
  const Mesh& m = M.mesh;
  for (auto& ps : M.psets) shapeMatrices(ps.layered ? ps.W : nullptr, ps.layered ? nullptr : ps.D, ps.M);
  std::fill(M.val.begin(), M.val.end(), 0.0);
  std::fill(rhs, rhs + M.ndof, 0.0);
  // a stacked-module stage assembles the born parts only (09-assembly.js:397-402)
  M.moduleStage = M.stage < 0 && !M.moduleConstraints.empty();
  ivec stageDofs;
  if (M.moduleStage) stageDofs = moduleStageSet(M, M.stage);
  else { M.actElem.clear(); M.actNode.clear(); }
  double K33[1089], f33[33], Kc[576], fc[24];
  for (int e = 0; e < m.ne; e++) {
    const bool born = M.groupStage[m.eGroup[e]] <= M.stage;
    if (M.moduleStage && !born) continue;
    const double scale = m.eScale[e] * (born ? 1 : UNBORN_SCALE);
    const PropSet& ps = M.psets[M.ePset[e]];
    const int i = m.eIJK[3 * e], j = m.eIJK[3 * e + 1], k = m.eIJK[3 * e + 2];
    const double hx = m.xs[i + 1] - m.xs[i], hy = m.ys[j + 1] - m.ys[j], hz = m.zs[k + 1] - m.zs[k];
    std::fill(f33, f33 + 33, 0.0);
    elementK33Fast(hx, hy, hz, ps.M, K33);
    bool hasF = ps.born;
    if (hasF) elementFth(hx, hy, hz, ps.layered ? ps.V : nullptr, ps.layered ? nullptr : ps.s0, f33);
    condense33(K33, hasF ? f33 : nullptr, Kc, fc, nullptr);
    for (int a = 0; a < 8; a++) {
      for (int b = 0; b < 8; b++) {
        const int kb = M.bmap[((size_t)e * 8 + a) * 8 + b];
        const size_t v = 9 * (size_t)kb;
        for (int p = 0; p < 3; p++) {
          const int r = (3 * a + p) * 24 + 3 * b;
          M.val[v + 3 * p] += scale * Kc[r]; M.val[v + 3 * p + 1] += scale * Kc[r + 1]; M.val[v + 3 * p + 2] += scale * Kc[r + 2];
        }
      }
      if (hasF) {
        const int n = m.conn[8 * e + a];
        rhs[3 * n] += scale * fc[3 * a]; rhs[3 * n + 1] += scale * fc[3 * a + 1]; rhs[3 * n + 2] += scale * fc[3 * a + 2];
      }
    }
  }
  if (!noConstraints) applyConstraints(M, rhs, M.moduleStage ? stageDofs : M.constraints);
  M.assembled = true;
}

// ---- multigrid (src/core/10-solver.js:12-715) -----------------------------------------
// chol3 :12-25
bool chol3(const double* A, double* L, double jit) {
  const double a00 = A[0] + jit, a10 = A[3], a11 = A[4] + jit, a20 = A[6], a21 = A[7], a22 = A[8] + jit;
  if (!(a00 > 0)) return false;
  const double l00 = std::sqrt(a00);
  const double l10 = a10 / l00, l20 = a20 / l00;
  const double d11 = a11 - l10 * l10;
  if (!(d11 > 0)) return false;
  const double l11 = std::sqrt(d11);
  const double l21 = (a21 - l20 * l10) / l11;
  const double d22 = a22 - l20 * l20 - l21 * l21;
  if (!(d22 > 0)) return false;
  L[0] = l00; L[1] = 0; L[2] = 0; L[3] = l10; L[4] = l11; L[5] = 0; L[6] = l20; L[7] = l21; L[8] = std::sqrt(d22);
  return true;
}

struct Prol { ivec ptr, idx; dvec W; };
struct Children { ivec ptr, idx, widx; };

struct Level {
  bool solid = true;
  int b = 3;
  int nx = 0, ny = 0, nz = 0, nn = 0;
  dvec xs, ys;
  ivec colStart;
  Pattern P;
  dvec val;
  // solid level
  ivec down;
  dvec colFact;            // 18 per node (solid)
  int colJitter = 0;
  // shell level
  ivec cfPtr; dvec cfData; // dense per-column factors
  dvec zref, zlo, zhi;
  // transfer to the next level
  Prol prol;
  Children children;
  ivec nodeAgg;
  ivec keepX, keepY; bool hasKeep = false;
  bool noHermite = false;
  // coarsest
  dvec band; int bandW = 0, bandBw = 0, denseN = 0, denseFixes = 0;
  // work vectors
  dvec r, dx, bvec, x, res;
};

// columnDownIndex :122-131
ivec columnDownIndex(const Pattern& P, const ivec& colStart) {
  ivec down(P.n, -1);
  for (size_t c = 0; c + 1 < colStart.size(); c++)
    for (int n = colStart[c] + 1; n < colStart[c + 1]; n++) down[n] = findBlock(P, n, n - 1);
  return down;
}

// factorColumns :31-68
void factorColumns(Level& L) {
  const Pattern& P = L.P; const double* val = L.val.data(); const int nn = P.n;
  L.colFact.assign((size_t)nn * 18, 0.0);
  double* F = L.colFact.data();
  double tmp[9], D[9];
  int jitter = 0;
  for (int n = 0; n < nn; n++) {
    const size_t dv = 9 * (size_t)P.diag[n];
    for (int q = 0; q < 9; q++) D[q] = val[dv + q];
    const size_t fo = 18 * (size_t)n;
    if (L.down[n] >= 0) {
      const size_t av = 9 * (size_t)L.down[n], lp = 18 * (size_t)(n - 1);
      for (int r = 0; r < 3; r++) {
        const double b0 = val[av + 3 * r], b1 = val[av + 3 * r + 1], b2 = val[av + 3 * r + 2];
        const double y0 = b0 / F[lp];
        const double y1 = (b1 - F[lp + 3] * y0) / F[lp + 4];
        const double y2 = (b2 - F[lp + 6] * y0 - F[lp + 7] * y1) / F[lp + 8];
        tmp[3 * r] = y0; tmp[3 * r + 1] = y1; tmp[3 * r + 2] = y2;
      }
      for (int q = 0; q < 9; q++) F[fo + 9 + q] = tmp[q];
      for (int r = 0; r < 3; r++) for (int c = 0; c < 3; c++)
        D[3 * r + c] -= tmp[3 * r] * tmp[3 * c] + tmp[3 * r + 1] * tmp[3 * c + 1] + tmp[3 * r + 2] * tmp[3 * c + 2];
    } else {
      for (int q = 0; q < 9; q++) F[fo + 9 + q] = 0;
    }
    double jit = 0;
    for (int t = 0; t < 8 && !chol3(D, F + fo, jit); t++) {
      jit = jit != 0 ? jit * 10 : 1e-10 * std::max(std::max(std::fabs(D[0]), std::fabs(D[4])), std::max(std::fabs(D[8]), 1e-300));
      jitter++;
    }
  }
  L.colJitter = jitter;
}

// solveColumn :71-104
void solveColumn(const Level& L, int n0, int n1, const double* r, double* x) {
  const double* F = L.colFact.data();
  for (int n = n0; n < n1; n++) {
    const size_t fo = 18 * (size_t)n;
    double b0 = r[3 * n], b1 = r[3 * n + 1], b2 = r[3 * n + 2];
    if (n > n0) {
      const double p0 = x[3 * n - 3], p1 = x[3 * n - 2], p2 = x[3 * n - 1];
      b0 -= F[fo + 9] * p0 + F[fo + 10] * p1 + F[fo + 11] * p2;
      b1 -= F[fo + 12] * p0 + F[fo + 13] * p1 + F[fo + 14] * p2;
      b2 -= F[fo + 15] * p0 + F[fo + 16] * p1 + F[fo + 17] * p2;
    }
    const double y0 = b0 / F[fo];
    const double y1 = (b1 - F[fo + 3] * y0) / F[fo + 4];
    const double y2 = (b2 - F[fo + 6] * y0 - F[fo + 7] * y1) / F[fo + 8];
    x[3 * n] = y0; x[3 * n + 1] = y1; x[3 * n + 2] = y2;
  }
  for (int n = n1 - 1; n >= n0; n--) {
    const size_t fo = 18 * (size_t)n;
    double b0 = x[3 * n], b1 = x[3 * n + 1], b2 = x[3 * n + 2];
    if (n + 1 < n1) {
      const size_t fn = 18 * (size_t)(n + 1);
      const double q0 = x[3 * n + 3], q1 = x[3 * n + 4], q2 = x[3 * n + 5];
      b0 -= F[fn + 9] * q0 + F[fn + 12] * q1 + F[fn + 15] * q2;
      b1 -= F[fn + 10] * q0 + F[fn + 13] * q1 + F[fn + 16] * q2;
      b2 -= F[fn + 11] * q0 + F[fn + 14] * q1 + F[fn + 17] * q2;
    }
    const double z2 = b2 / F[fo + 8];
    const double z1 = (b1 - F[fo + 7] * z2) / F[fo + 4];
    const double z0 = (b0 - F[fo + 3] * z1 - F[fo + 6] * z2) / F[fo];
    x[3 * n] = z0; x[3 * n + 1] = z1; x[3 * n + 2] = z2;
  }
}

// coarseLines :171-177
ivec coarseLines(int n, const ivec* keep) {
  std::set<int> s;
  for (int i = 0; i < n; i += 2) s.insert(i);
  s.insert(n - 1);
  if (keep) for (int k : *keep) if (k >= 0 && k < n) s.insert(k);
  return ivec(s.begin(), s.end());
}

// transposeProl :180-187
Children transposeProl(const Prol& prol, int nnc) {
  Children ch; ch.ptr.assign(nnc + 1, 0);
  for (size_t q = 0; q < prol.idx.size(); q++) ch.ptr[prol.idx[q] + 1]++;
  for (int c = 0; c < nnc; c++) ch.ptr[c + 1] += ch.ptr[c];
  ch.idx.assign(prol.idx.size(), 0); ch.widx.assign(prol.idx.size(), 0);
  ivec fill(ch.ptr.begin(), ch.ptr.begin() + nnc);
  for (size_t f = 0; f + 1 < prol.ptr.size(); f++) for (int q = prol.ptr[f]; q < prol.ptr[f + 1]; q++) {
    const int c = prol.idx[q]; ch.idx[fill[c]] = (int)f; ch.widx[fill[c]] = q; fill[c]++;
  }
  return ch;
}

// galerkinProduct :193-245
void galerkinProduct(Level& L, Level& C) {
  const Children& ch = C.children; const Prol& prol = L.prol;
  const int bf = L.b, bc = C.b, bfc = bf * bc, bcc = bc * bc, bff = bf * bf;
  const Pattern& P = L.P; const double* val = L.val.data(); const int nnc = C.nn; const double* W = prol.W.data();
  ivec mark(nnc, -1);
  dvec acc((size_t)nnc * bcc, 0.0);
  ivec touched;
  Pattern CP; CP.n = nnc; CP.rowPtr.assign(nnc + 1, 0);
  ivec cols; dvec vals;
  cols.reserve((size_t)27 * nnc); vals.reserve((size_t)27 * nnc * bcc);
  double T[36];
  for (int I = 0; I < nnc; I++) {
    touched.clear();
    for (int q = ch.ptr[I]; q < ch.ptr[I + 1]; q++) {
      const int i = ch.idx[q]; const size_t wi = (size_t)ch.widx[q] * bfc;
      for (int k = P.rowPtr[i]; k < P.rowPtr[i + 1]; k++) {
        const int j = P.col[k]; const size_t v = (size_t)bff * k;
        for (int p = prol.ptr[j]; p < prol.ptr[j + 1]; p++) {
          const int J = prol.idx[p]; const size_t wj = (size_t)p * bfc;
          if (mark[J] != I) { mark[J] = I; touched.push_back(J); std::fill(acc.begin() + (size_t)bcc * J, acc.begin() + (size_t)bcc * J + bcc, 0.0); }
          for (int r = 0; r < bf; r++) {
            const size_t vr = v + r * bf;
            for (int c = 0; c < bc; c++) {
              double sum = 0;
              for (int t = 0; t < bf; t++) sum += val[vr + t] * W[wj + t * bc + c];
              T[r * bc + c] = sum;
            }
          }
          const size_t a = (size_t)bcc * J;
          for (int r = 0; r < bc; r++) for (int c = 0; c < bc; c++) {
            double sum = 0;
            for (int t = 0; t < bf; t++) sum += W[wi + t * bc + r] * T[t * bc + c];
            acc[a + r * bc + c] += sum;
          }
        }
      }
    }
    std::sort(touched.begin(), touched.end());
    CP.rowPtr[I + 1] = CP.rowPtr[I] + (int)touched.size();
    for (int J : touched) { cols.push_back(J); vals.insert(vals.end(), acc.begin() + (size_t)bcc * J, acc.begin() + (size_t)bcc * J + bcc); }
  }
  CP.col = cols; CP.nb = (int)cols.size();
  CP.diag.assign(nnc, 0);
  for (int I = 0; I < nnc; I++) for (int k = CP.rowPtr[I]; k < CP.rowPtr[I + 1]; k++) if (CP.col[k] == I) { CP.diag[I] = k; break; }
  C.P = CP; C.val = vals;
}

// shellWeights :337-353
void shellWeights(Level& L, const Level& C, const dvec& coords, const double* s) {
  const int nn = L.nn;
  int ne = 0;
  for (int n = 0; n < nn; n++) if (L.nodeAgg[n] >= 0) ne++;
  L.prol.ptr.assign(nn + 1, 0); L.prol.idx.assign(ne, 0); L.prol.W.assign((size_t)ne * 18, 0.0);
  for (int n = 0, q = 0; n < nn; n++) {
    L.prol.ptr[n + 1] = L.prol.ptr[n];
    if (L.nodeAgg[n] < 0) continue;
    L.prol.ptr[n + 1]++; L.prol.idx[q] = L.nodeAgg[n];
    const double zp = coords[3 * n + 2] - C.zref[L.nodeAgg[n]];
    double* W = L.prol.W.data() + 18 * (size_t)q++;
    W[0] = 1 / s[3 * n]; W[4] = zp / s[3 * n];
    W[7] = 1 / s[3 * n + 1]; W[9] = -zp / s[3 * n + 1];
    W[14] = 1 / s[3 * n + 2]; W[17] = zp / s[3 * n + 2];
  }
}


// The reference reads cellElems at the flat index (i*ncy + j)*ncz + k for a node
// column (i, j); at j = ny-1 that index belongs to cell (i+1, 0, k) and at
// i = nx-1 it lies past the array (undefined in JavaScript, i.e. no element).
// Both effects are reproduced here (10-solver.js:270-287).
int cellElemAt(const Mesh& mesh, long c, int q) {
  const long idx = 2 * c + q;
  if (idx < 0 || idx >= (long)mesh.cellElems.size()) return -1;
  return mesh.cellElems[idx];
}

// buildShellLevel :260-334; s = Jacobi scaling. act (stacked-module stages, :262-266): when actElem is
// not empty, the elements not born in the stage count as void and the nodes they alone touch stay
// out of every aggregate
void buildShellLevel(Level& L, Level& C, const Mesh& mesh, const double* s, const char* mergeSingles,
                     const std::vector<uint8_t>& actElem, const std::vector<uint8_t>& actNode) {
  const bool act = !actElem.empty();
  auto elemOn = [&](int e) { return e >= 0 && (!act || actElem[e]); };
  const int nx = L.nx, ny = L.ny, nz = L.nz, ncy = ny - 1, ncz = nz - 1;
  const int ncol = nx * ny;
  C.colStart.assign(ncol + 1, 0);
  L.nodeAgg.assign(L.nn, -1);
  dvec zlo, zhi, zref;
  int na = 0;
  auto isCompliant = [&](int i, int j, int k) {
    const long c = ((long)i * ncy + j) * ncz + k;
    bool any = false, stiff = false;
    for (int q = 0; q < 2; q++) {
      const int e = cellElemAt(mesh, c, q);
      if (!elemOn(e)) continue;
      any = true;
      if (!is_compliant_part(mesh.ePart[e])) stiff = true;
    }
    return any && !stiff;
  };
  auto hasElem = [&](int i, int j, int k) {
    const long c = ((long)i * ncy + j) * ncz + k;
    return elemOn(cellElemAt(mesh, c, 0)) || elemOn(cellElemAt(mesh, c, 1));
  };
  auto elemClass = [&](int i, int j, int k) -> int {
    return (k < 0 || k >= ncz || !hasElem(i, j, k)) ? 0 : (isCompliant(i, j, k) ? 1 : 2);
  };
  struct NodeRec { int n, k; double z; };
  const std::string merge = mergeSingles ? mergeSingles : "none";
  for (int c = 0; c < ncol; c++) {
    C.colStart[c] = na;
    const int i = c / ny, j = c % ny;
    std::vector<std::vector<NodeRec>> runs;
    int cur = -1, prevK = -2, prevType = 0;   // cur: index of the current run, -1 = none
    for (int k = 0; k < nz; k++) {
      const int n = mesh.nodeId[(size_t)c * nz + k];
      if (n < 0 || (act && !actNode[n])) { cur = -1; prevK = -2; continue; }
      const int below = elemClass(i, j, k - 1), above = elemClass(i, j, k);
      const int type = (below == 2 || above == 2) ? 2 : 1;
      bool joined = false;
      if (cur >= 0 && prevK == k - 1 && below != 0) joined = below == 2 || (type == 1 && prevType == 1);
      if (!joined) { runs.emplace_back(); cur = (int)runs.size() - 1; }
      runs[cur].push_back({n, k, mesh.coords[3 * (size_t)n + 2]});
      prevK = k; prevType = type;
    }
    if (merge != "none") {
      for (int r = 0; r < (int)runs.size(); r++) {
        if (runs[r].size() != 1 || runs.size() < 2) continue;
        const int t = merge == "below" ? (r > 0 ? r - 1 : r + 1) : (r + 1 < (int)runs.size() ? r + 1 : r - 1);
        if (t < r) runs[t].push_back(runs[r][0]); else runs[t].insert(runs[t].begin(), runs[r][0]);
        runs.erase(runs.begin() + r); r--;
      }
    }
    for (auto& run : runs) {
      double zs = 0;
      for (auto& o : run) { L.nodeAgg[o.n] = na; zs += o.z; }
      zlo.push_back(run[0].z); zhi.push_back(run.back().z); zref.push_back(zs / run.size());
      na++;
    }
  }
  C.colStart[ncol] = na;
  C.solid = false; C.b = 6; C.nx = nx; C.ny = ny; C.nn = na; C.xs = L.xs; C.ys = L.ys;
  C.zref = zref; C.zlo = zlo; C.zhi = zhi;
  C.keepX = L.keepX; C.keepY = L.keepY; C.hasKeep = L.hasKeep;
  shellWeights(L, C, mesh.coords, s);
  C.children = transposeProl(L.prol, na);
  galerkinProduct(L, C);
}

// hermitePair :356-363
void hermitePair(double t, double h, bool alongY, double* WA, double* WB) {
  std::fill(WA, WA + 36, 0.0); std::fill(WB, WB + 36, 0.0);
  for (int d = 0; d < 6; d++) { WA[d * 6 + d] = 1 - t; WB[d * 6 + d] = t; }
  const double h00 = 2 * t * t * t - 3 * t * t + 1, h10 = t * t * t - 2 * t * t + t, h01 = -2 * t * t * t + 3 * t * t, h11 = t * t * t - t * t;
  WA[2 * 6 + 2] = h00; WB[2 * 6 + 2] = h01;
  if (alongY) { WA[2 * 6 + 3] = h * h10; WB[2 * 6 + 3] = h * h11; }
  else { WA[2 * 6 + 4] = -h * h10; WB[2 * 6 + 4] = -h * h11; }
}

// rbmShift :366-373
void rbmShift(double dz, double* M) {
  std::fill(M, M + 36, 0.0);
  for (int d = 0; d < 6; d++) M[d * 7] = 1;
  M[0 * 6 + 4] = dz; M[1 * 6 + 3] = -dz; M[2 * 6 + 5] = dz;
}

// mul66 :375-378
void mul66(const double* A, const double* B, double* C) {
  double T[36];
  for (int i = 0; i < 6; i++) for (int j = 0; j < 6; j++) { double s = 0; for (int k = 0; k < 6; k++) s += A[i * 6 + k] * B[k * 6 + j]; T[i * 6 + j] = s; }
  std::memcpy(C, T, sizeof(T));
}

// matchAggregate :381-389
int matchAggregate(const Level& C, int col, double zlo, double zhi, double zref) {
  int best = -1; double bo = 0;
  for (int a = C.colStart[col]; a < C.colStart[col + 1]; a++) {
    const double ov = std::min(zhi, C.zhi[a]) - std::max(zlo, C.zlo[a]);
    const double score = ov > 0 ? ov + 1e-9 : (zref >= C.zlo[a] - 1e-9 && zref <= C.zhi[a] + 1e-9 ? 1e-9 : -1);
    if (score > bo) { bo = score; best = a; }
  }
  return best;
}

// buildCoarseShellLevel :396-471
void buildCoarseShellLevel(Level& L, Level& C) {
  const ivec cx = coarseLines(L.nx, L.hasKeep ? &L.keepX : nullptr), cy = coarseLines(L.ny, L.hasKeep ? &L.keepY : nullptr);
  const int nxc = (int)cx.size(), nyc = (int)cy.size();
  dvec xsc(nxc), ysc(nyc);
  for (int I = 0; I < nxc; I++) xsc[I] = L.xs[cx[I]];
  for (int J = 0; J < nyc; J++) ysc[J] = L.ys[cy[J]];
  C.colStart.assign((size_t)nxc * nyc + 1, 0);
  C.zlo.clear(); C.zhi.clear(); C.zref.clear();
  int na = 0;
  for (int I = 0; I < nxc; I++) for (int J = 0; J < nyc; J++) {
    C.colStart[I * nyc + J] = na;
    const int c = cx[I] * L.ny + cy[J];
    for (int a = L.colStart[c]; a < L.colStart[c + 1]; a++) { C.zlo.push_back(L.zlo[a]); C.zhi.push_back(L.zhi[a]); C.zref.push_back(L.zref[a]); na++; }
  }
  C.colStart[(size_t)nxc * nyc] = na;
  C.solid = false; C.b = 6; C.nx = nxc; C.ny = nyc; C.xs = xsc; C.ys = ysc; C.nn = na;
  C.hasKeep = L.hasKeep;
  if (L.hasKeep) {
    C.keepX.clear(); C.keepY.clear();
    for (int i : L.keepX) { auto it = std::find(cx.begin(), cx.end(), i); if (it != cx.end()) C.keepX.push_back((int)(it - cx.begin())); }
    for (int j : L.keepY) { auto it = std::find(cy.begin(), cy.end(), j); if (it != cy.end()) C.keepY.push_back((int)(it - cy.begin())); }
  }
  struct Loc { int I0, I1; double t, h; };
  auto locate = [](const ivec& lines, const dvec& coords, int i, double x) {
    int I0 = 0;
    while (I0 + 1 < (int)lines.size() && lines[I0 + 1] <= i) I0++;
    if (lines[I0] == i) return Loc{I0, -1, 0, 0};
    return Loc{I0, I0 + 1, (x - coords[I0]) / (coords[I0 + 1] - coords[I0]), coords[I0 + 1] - coords[I0]};
  };
  L.prol.ptr.assign(L.nn + 1, 0);
  ivec idx; dvec Wl;
  double WL[36], WR[36], WB[36], WT[36], tmp[36], sh[36], tmp2[36];
  for (int i = 0; i < L.nx; i++) {
    const Loc px = locate(cx, xsc, i, L.xs[i]);
    for (int j = 0; j < L.ny; j++) {
      const Loc py = locate(cy, ysc, j, L.ys[j]);
      const int c = i * L.ny + j;
      for (int f = L.colStart[c]; f < L.colStart[c + 1]; f++) {
        auto get = [&](int I, int J) { return matchAggregate(C, I * nyc + J, L.zlo[f], L.zhi[f], L.zref[f]); };
        ivec xC = px.I1 < 0 ? ivec{px.I0} : ivec{px.I0, px.I1};
        ivec yC = py.I1 < 0 ? ivec{py.I0} : ivec{py.I0, py.I1};
        std::map<std::pair<int, int>, int> par;
        bool complete = true;
        for (int I : xC) for (int J : yC) { const int a = get(I, J); par[{I, J}] = a; if (a < 0) complete = false; }
        int count = 0;
        auto push = [&](int I, int J, const double* W) {
          const int a = par[{I, J}];
          rbmShift(L.zref[f] - C.zref[a], sh);
          mul66(W, sh, tmp2);
          idx.push_back(a); Wl.insert(Wl.end(), tmp2, tmp2 + 36); count++;
        };
        if (complete) {
          if (px.I1 >= 0) hermitePair(px.t, L.noHermite ? 0 : px.h, false, WL, WR);
          if (py.I1 >= 0) hermitePair(py.t, L.noHermite ? 0 : py.h, true, WB, WT);
          if (px.I1 < 0 && py.I1 < 0) { double W[36] = {0}; for (int d = 0; d < 6; d++) W[d * 7] = 1; push(px.I0, py.I0, W); }
          else if (py.I1 < 0) { push(px.I0, py.I0, WL); push(px.I1, py.I0, WR); }
          else if (px.I1 < 0) { push(px.I0, py.I0, WB); push(px.I0, py.I1, WT); }
          else {
            mul66(WB, WL, tmp); push(px.I0, py.I0, tmp); mul66(WB, WR, tmp); push(px.I1, py.I0, tmp);
            mul66(WT, WL, tmp); push(px.I0, py.I1, tmp); mul66(WT, WR, tmp); push(px.I1, py.I1, tmp);
          }
        } else {
          dvec wx = px.I1 < 0 ? dvec{1} : dvec{1 - px.t, px.t}, wy = py.I1 < 0 ? dvec{1} : dvec{1 - py.t, py.t};
          double sum = 0;
          struct Ex { int I, J; double w; };
          std::vector<Ex> ex;
          for (size_t a = 0; a < xC.size(); a++) for (size_t b = 0; b < yC.size(); b++) {
            const int ag = par[{xC[a], yC[b]}]; const double w = wx[a] * wy[b];
            if (ag >= 0 && w > 0) { ex.push_back({xC[a], yC[b], w}); sum += w; }
          }
          for (auto& e : ex) { double W[36] = {0}; for (int d = 0; d < 6; d++) W[d * 7] = e.w / sum; push(e.I, e.J, W); }
        }
        L.prol.ptr[f + 1] = count;
      }
    }
  }
  for (int f = 0; f < L.nn; f++) L.prol.ptr[f + 1] += L.prol.ptr[f];
  L.prol.idx = idx; L.prol.W = Wl;
  C.children = transposeProl(L.prol, na);
  galerkinProduct(L, C);
}

// factorShellColumns :474-494
void factorShellColumns(Level& L) {
  const int b = L.b, ncol = (int)L.colStart.size() - 1, bb = b * b;
  L.cfPtr.assign(ncol + 1, 0);
  for (int c = 0; c < ncol; c++) { const int m = (L.colStart[c + 1] - L.colStart[c]) * b; L.cfPtr[c + 1] = L.cfPtr[c] + m * m; }
  L.cfData.assign(L.cfPtr[ncol], 0.0);
  int fixes = 0;
  for (int c = 0; c < ncol; c++) {
    const int n0 = L.colStart[c], n1 = L.colStart[c + 1], m = (n1 - n0) * b;
    if (!m) continue;
    double* A = L.cfData.data() + L.cfPtr[c];
    for (int n = n0; n < n1; n++) for (int k = L.P.rowPtr[n]; k < L.P.rowPtr[n + 1]; k++) {
      const int j = L.P.col[k];
      if (j < n0 || j >= n1) continue;
      const size_t v = (size_t)bb * k;
      for (int p = 0; p < b; p++) for (int q = 0; q < b; q++) A[((n - n0) * b + p) * m + (j - n0) * b + q] = L.val[v + p * b + q];
    }
    fixes += cholDense(A, m, 1e-12);
  }
  L.colJitter = fixes;
}

// columnSweep :512-555
void columnSweep(Level& L, const double* bvec, double* x, bool backward) {
  const Pattern& P = L.P; const double* val = L.val.data(); const int ncol = (int)L.colStart.size() - 1;
  double* r = L.r.data(); double* dx = L.dx.data();
  for (int cc = 0; cc < ncol; cc++) {
    const int c = backward ? ncol - 1 - cc : cc;
    const int n0 = L.colStart[c], n1 = L.colStart[c + 1];
    if (n1 == n0) continue;
    if (L.solid) {
      for (int n = n0; n < n1; n++) {
        double s0 = bvec[3 * n], s1 = bvec[3 * n + 1], s2 = bvec[3 * n + 2];
        for (int k = P.rowPtr[n]; k < P.rowPtr[n + 1]; k++) {
          const int j = P.col[k]; const size_t v = 9 * (size_t)k;
          const double xj0 = x[3 * j], xj1 = x[3 * j + 1], xj2 = x[3 * j + 2];
          s0 -= val[v] * xj0 + val[v + 1] * xj1 + val[v + 2] * xj2;
          s1 -= val[v + 3] * xj0 + val[v + 4] * xj1 + val[v + 5] * xj2;
          s2 -= val[v + 6] * xj0 + val[v + 7] * xj1 + val[v + 8] * xj2;
        }
        r[3 * n] = s0; r[3 * n + 1] = s1; r[3 * n + 2] = s2;
      }
      solveColumn(L, n0, n1, r, dx);
      for (int q = 3 * n0; q < 3 * n1; q++) x[q] += dx[q];
    } else {
      for (int n = n0; n < n1; n++) {
        double s[6];
        for (int t = 0; t < 6; t++) s[t] = bvec[6 * n + t];
        for (int k = P.rowPtr[n]; k < P.rowPtr[n + 1]; k++) {
          const int j = P.col[k]; const size_t v = 36 * (size_t)k; const int o = 6 * j;
          for (int t = 0; t < 6; t++) {
            const double* vr = val + v + 6 * t;
            s[t] -= vr[0] * x[o] + vr[1] * x[o + 1] + vr[2] * x[o + 2] + vr[3] * x[o + 3] + vr[4] * x[o + 4] + vr[5] * x[o + 5];
          }
        }
        for (int t = 0; t < 6; t++) r[6 * n + t] = s[t];
      }
      const int m = (n1 - n0) * 6;
      cholSolveDenseOff(L.cfData.data() + L.cfPtr[c], m, r + 6 * n0);
      for (int q = 6 * n0; q < 6 * n1; q++) x[q] += r[q];
    }
  }
}

// factorCoarsest :562-600
void factorCoarsest(Level& L) {
  const int b = L.b, n = b * L.nn, bb = b * b;
  int bw = 0;
  for (int i = 0; i < L.nn; i++) for (int k = L.P.rowPtr[i]; k < L.P.rowPtr[i + 1]; k++) bw = std::max(bw, std::abs(L.P.col[k] - i));
  bw = (bw + 1) * b - 1;
  const int w = bw + 1;
  L.band.assign((size_t)n * w, 0.0);
  double* A = L.band.data();
  for (int i = 0; i < L.nn; i++) for (int k = L.P.rowPtr[i]; k < L.P.rowPtr[i + 1]; k++) {
    const int j = L.P.col[k]; const size_t v = (size_t)bb * k;
    if (j > i) continue;
    for (int p = 0; p < b; p++) for (int q = 0; q < b; q++) {
      const int r = b * i + p, c = b * j + q;
      if (c <= r) A[(size_t)r * w + (c - r + bw)] = L.val[v + p * b + q];
    }
  }
  double dmax = 0;
  for (int i = 0; i < n; i++) dmax = std::max(dmax, std::fabs(A[(size_t)i * w + bw]));
  const double jitter = 1e-12 * (dmax != 0 ? dmax : 1);
  int fixes = 0;
  for (int j = 0; j < n; j++) {
    double d = A[(size_t)j * w + bw];
    const int k0 = std::max(0, j - bw);
    for (int k = k0; k < j; k++) { const double l = A[(size_t)j * w + (k - j + bw)]; d -= l * l; }
    if (!(d > jitter)) { d = std::max(std::fabs(d), jitter); fixes++; }
    const double ljj = std::sqrt(d);
    A[(size_t)j * w + bw] = ljj;
    const double inv = 1 / ljj;
    const int iend = std::min(n, j + bw + 1);
    for (int i = j + 1; i < iend; i++) {
      double sum = A[(size_t)i * w + (j - i + bw)];
      const int kk0 = std::max(k0, i - bw);
      for (int k = kk0; k < j; k++) sum -= A[(size_t)i * w + (k - i + bw)] * A[(size_t)j * w + (k - j + bw)];
      A[(size_t)i * w + (j - i + bw)] = sum * inv;
    }
  }
  L.denseFixes = fixes; L.bandW = w; L.bandBw = bw; L.denseN = n;
}

// solveCoarsest :603-617
void solveCoarsest(const Level& L, double* x) {
  const double* A = L.band.data(); const int w = L.bandW, bw = L.bandBw, n = L.denseN;
  for (int i = 0; i < n; i++) {
    double sum = x[i];
    const int k0 = std::max(0, i - bw);
    for (int k = k0; k < i; k++) sum -= A[(size_t)i * w + (k - i + bw)] * x[k];
    x[i] = sum / A[(size_t)i * w + bw];
  }
  for (int i = n - 1; i >= 0; i--) {
    double sum = x[i];
    const int kend = std::min(n, i + bw + 1);
    for (int k = i + 1; k < kend; k++) sum -= A[(size_t)k * w + (i - k + bw)] * x[k];
    x[i] = sum / A[(size_t)i * w + bw];
  }
}

// Preconditioner interface
struct Precond {
  virtual ~Precond() {}
  virtual void apply(const double* r, double* z) = 0;
  double setupMs = 0;
};

// MultigridPC :620-715
struct MultigridPC : Precond {
  std::vector<std::unique_ptr<Level>> levels;
  int pre = 2, post = 2;
  bool symmetric = false;
  int colJitter = 0, shellJitter = 0;

  MultigridPC(const Mesh& mesh, const Pattern& P, const dvec& val, const dvec& s, const std::vector<uint8_t>& actElem,
              const std::vector<uint8_t>& actNode) {
    const double t0 = now_ms();
    auto fine = std::make_unique<Level>();
    fine->solid = true; fine->b = 3; fine->nx = mesh.nx; fine->ny = mesh.ny; fine->nz = mesh.nz; fine->nn = mesh.nn;
    fine->xs = mesh.xs; fine->ys = mesh.ys; fine->colStart = mesh.colStart; fine->P = P; fine->val = val;
    fine->down = columnDownIndex(P, fine->colStart);
    fine->r.assign(3 * (size_t)mesh.nn, 0.0); fine->dx.assign(3 * (size_t)mesh.nn, 0.0);
    if (mesh.hasFeatures) { fine->keepX = mesh.featureX; fine->keepY = mesh.featureY; fine->hasKeep = true; }
    factorColumns(*fine);
    colJitter = fine->colJitter;
    levels.push_back(std::move(fine));
    auto lv = std::make_unique<Level>();
    buildShellLevel(*levels[0], *lv, mesh, s.data(), "below", actElem, actNode);
    levels.push_back(std::move(lv));
    for (int guard = 0; guard < 20; guard++) {
      Level& cur = *levels.back();
      factorShellColumns(cur);
      shellJitter += cur.colJitter;
      const int ncol = cur.nx * cur.ny, ndof = cur.b * cur.nn;
      if (ncol <= MG_COARSEST_COLS || ndof <= MG_COARSEST_DOF || (cur.nx <= 2 && cur.ny <= 2)) break;
      const int ncx = (int)coarseLines(cur.nx, cur.hasKeep ? &cur.keepX : nullptr).size();
      const int ncy = (int)coarseLines(cur.ny, cur.hasKeep ? &cur.keepY : nullptr).size();
      if (ncx * ncy > MG_MIN_COARSENING * ncol) break;
      auto nl = std::make_unique<Level>();
      buildCoarseShellLevel(cur, *nl);
      levels.push_back(std::move(nl));
    }
    factorCoarsest(*levels.back());
    for (auto& l : levels) {
      const size_t n = (size_t)l->b * l->nn;
      l->bvec.assign(n, 0.0); l->x.assign(n, 0.0); l->res.assign(n, 0.0);
      if (l->r.size() != n) l->r.assign(n, 0.0);
      if (l->dx.size() != n) l->dx.assign(n, 0.0);
    }
    setupMs = now_ms() - t0;
  }

  void cycleOnce(size_t li, const double* bvec, double* x) {
    Level& lv = *levels[li];
    const size_t n = (size_t)lv.b * lv.nn;
    std::fill(x, x + n, 0.0);
    if (li == levels.size() - 1) { std::copy(bvec, bvec + n, x); solveCoarsest(lv, x); return; }
    for (int s = 0; s < pre; s++) { columnSweep(lv, bvec, x, false); if (symmetric) columnSweep(lv, bvec, x, true); }
    double* res = lv.res.data();
    blockMatVec(lv.P, lv.val.data(), lv.b, x, res);
    for (size_t i = 0; i < n; i++) res[i] = bvec[i] - res[i];
    Level& co = *levels[li + 1];
    const Prol& prol = lv.prol;
    const int bf = lv.b, bc = co.b, bfc = bf * bc;
    double* rc = co.bvec.data();
    std::fill(co.bvec.begin(), co.bvec.end(), 0.0);
    for (int f = 0; f < lv.nn; f++) {
      for (int q = prol.ptr[f]; q < prol.ptr[f + 1]; q++) {
        const int c = prol.idx[q]; const size_t w = (size_t)bfc * q;
        for (int a = 0; a < bc; a++) { double s = 0; for (int p = 0; p < bf; p++) s += prol.W[w + p * bc + a] * res[bf * f + p]; rc[bc * c + a] += s; }
      }
    }
    cycleOnce(li + 1, rc, co.x.data());
    const double* ec = co.x.data();
    for (int f = 0; f < lv.nn; f++) {
      for (int q = prol.ptr[f]; q < prol.ptr[f + 1]; q++) {
        const int c = prol.idx[q]; const size_t w = (size_t)bfc * q;
        for (int p = 0; p < bf; p++) { double s = 0; for (int a = 0; a < bc; a++) s += prol.W[w + p * bc + a] * ec[bc * c + a]; x[bf * f + p] += s; }
      }
    }
    for (int s = 0; s < post; s++) { if (symmetric) columnSweep(lv, bvec, x, false); columnSweep(lv, bvec, x, true); }
  }

  void apply(const double* r, double* z) override { cycleOnce(0, r, z); }
};

// ICPC :719-800
struct ICPC : Precond {
  int n = 0; ivec rowPtr, col; dvec v; double shift = 0;
  ICPC(const Pattern& P, const dvec& val) {
    const double t0 = now_ms();
    n = 3 * P.n;
    rowPtr.assign(n + 1, 0);
    for (int i = 0; i < P.n; i++) for (int p = 0; p < 3; p++) {
      int c = 0;
      for (int k = P.rowPtr[i]; k < P.rowPtr[i + 1]; k++) { const int j = P.col[k]; if (j > i) c += 3; else if (j == i) c += 3 - p; }
      rowPtr[3 * i + p + 1] = rowPtr[3 * i + p] + c;
    }
    col.assign(rowPtr[n], 0); dvec v0(rowPtr[n], 0.0);
    for (int i = 0; i < P.n; i++) for (int p = 0; p < 3; p++) {
      int w = rowPtr[3 * i + p];
      for (int k = P.rowPtr[i]; k < P.rowPtr[i + 1]; k++) {
        const int j = P.col[k];
        if (j < i) continue;
        for (int q = (j == i ? p : 0); q < 3; q++) { col[w] = 3 * j + q; v0[w] = val[9 * (size_t)k + 3 * p + q]; w++; }
      }
    }
    double sh = 0;
    bool ok = false;
    for (int attempt = 0; attempt < 8; attempt++) {
      v = v0;
      if (sh > 0) for (int i = 0; i < n; i++) v[rowPtr[i]] *= 1 + sh;
      if (factor()) { shift = sh; ok = true; break; }
      sh = sh == 0 ? IC_SHIFT0 : sh * 10;
      if (sh > IC_SHIFT_MAX) sh = IC_SHIFT_MAX;
    }
    if (!ok) throw std::runtime_error("IC(0) failed even with the maximum diagonal shift");
    setupMs = now_ms() - t0;
  }
  bool factor() {
    for (int i = 0; i < n; i++) {
      const double d = v[rowPtr[i]];
      if (!(d > 0)) return false;
      const double uii = std::sqrt(d);
      v[rowPtr[i]] = uii;
      for (int k = rowPtr[i] + 1; k < rowPtr[i + 1]; k++) v[k] /= uii;
      for (int k1 = rowPtr[i] + 1; k1 < rowPtr[i + 1]; k1++) {
        const int j1 = col[k1]; const double u1 = v[k1];
        int kk = rowPtr[j1]; const int kend = rowPtr[j1 + 1];
        for (int k2 = k1; k2 < rowPtr[i + 1]; k2++) {
          const int j2 = col[k2];
          while (kk < kend && col[kk] < j2) kk++;
          if (kk < kend && col[kk] == j2) v[kk] -= u1 * v[k2];
        }
      }
    }
    return true;
  }
  void apply(const double* r, double* z) override {
    std::copy(r, r + n, z);
    for (int i = 0; i < n; i++) {
      const double yi = z[i] / v[rowPtr[i]];
      z[i] = yi;
      for (int k = rowPtr[i] + 1; k < rowPtr[i + 1]; k++) z[col[k]] -= v[k] * yi;
    }
    for (int i = n - 1; i >= 0; i--) {
      double s = z[i];
      for (int k = rowPtr[i] + 1; k < rowPtr[i + 1]; k++) s -= v[k] * z[col[k]];
      z[i] = s / v[rowPtr[i]];
    }
  }
};

// ---- LinearSolver (10-solver.js:826-1043) --------------------------------------------
struct PcgResult { int iters = 0; double relres = 0; bool converged = false; double iters0 = 0; };

struct SolveInfo {
  int iters = 0; double relres = 0; int converged = 0; double iters0 = 0;
  double ms = 0, pcMs = 0; int precond = 0; int rebuilt = 0; int warm = 0; int fallback = 0;
  int colJitter = 0, shellJitter = 0, levels = 0;
};

struct LinearSolver {
  Model* model;
  int precondKind = 0;   // 0 = MG, 1 = IC(0)
  double tol = PCG_TOL; int maxit = PCG_MAXIT; int warmMax = WARM_START_MAX;
  dvec s, r, z, p, q, bs, x;
  std::unique_ptr<Precond> pc;
  int pcKind = -1;
  double ratePerDecade = 0;
  bool needRebuild = true;
  long pcKey = -1;
  std::vector<dvec> basis;

  explicit LinearSolver(Model* m) : model(m) {
    const size_t n = m->ndof;
    s.assign(n, 0.0); r.assign(n, 0.0); z.assign(n, 0.0); p.assign(n, 0.0); q.assign(n, 0.0); bs.assign(n, 0.0); x.assign(n, 0.0);
  }

  // _scale :852-866
  void scale() {
    const Pattern& P = model->pattern; double* val = model->val.data();
    for (int i = 0; i < P.n; i++) {
      const size_t v = 9 * (size_t)P.diag[i];
      s[3 * i] = 1 / std::sqrt(std::max(val[v], 1e-300));
      s[3 * i + 1] = 1 / std::sqrt(std::max(val[v + 4], 1e-300));
      s[3 * i + 2] = 1 / std::sqrt(std::max(val[v + 8], 1e-300));
    }
    for (int i = 0; i < P.n; i++) for (int k = P.rowPtr[i]; k < P.rowPtr[i + 1]; k++) {
      const int j = P.col[k]; const size_t v = 9 * (size_t)k;
      for (int pp = 0; pp < 3; pp++) for (int qq = 0; qq < 3; qq++) val[v + 3 * pp + qq] *= s[3 * i + pp] * s[3 * j + qq];
    }
  }

  // _buildPC :868-882 (a new hierarchy each time, over the active set of a stacked-module stage)
  double buildPC(int kind) {
    const double t0 = now_ms();
    if (kind == 0) pc.reset(new MultigridPC(model->mesh, model->pattern, model->val, s, model->actElem, model->actNode));
    else pc.reset(new ICPC(model->pattern, model->val));
    pcKind = kind;
    needRebuild = false;
    return now_ms() - t0;
  }

  // _warmStart :885-915
  void warmStart(const dvec& fs, dvec& xv) {
    const int m = (int)basis.size();
    std::fill(xv.begin(), xv.end(), 0.0);
    if (!m) return;
    const size_t n = model->ndof;
    std::vector<dvec> KV;
    dvec tmp(n), tmp2(n);
    for (int i = 0; i < m; i++) {
      const dvec& v = basis[i];
      for (size_t qq = 0; qq < n; qq++) tmp[qq] = v[qq] / s[qq];
      fullMatVec(model->pattern, model->val.data(), tmp.data(), tmp2.data());
      dvec kv(n);
      for (size_t qq = 0; qq < n; qq++) kv[qq] = tmp2[qq] / s[qq];
      KV.push_back(kv);
    }
    dvec A((size_t)m * m), b(m);
    for (int i = 0; i < m; i++) {
      double bi = 0;
      for (size_t qq = 0; qq < n; qq++) bi += basis[i][qq] * fs[qq] / s[qq];
      b[i] = bi;
      for (int j = 0; j < m; j++) A[i * m + j] = dot(basis[i], KV[j]);
    }
    for (int i = 0; i < m; i++) for (int j = i + 1; j < m; j++) { const double v = 0.5 * (A[i * m + j] + A[j * m + i]); A[i * m + j] = A[j * m + i] = v; }
    dvec c(m);
    if (!solveDense(A.data(), m, b.data(), c.data())) return;
    for (int i = 0; i < m; i++) if (!std::isfinite(c[i])) return;
    for (int i = 0; i < m; i++) axpy(c[i], basis[i], xv);
    for (size_t qq = 0; qq < n; qq++) xv[qq] /= s[qq];
  }

  // _storeSolution :917-926
  void storeSolution(const dvec& u) {
    dvec v = u;
    for (auto& b : basis) axpy(-dot(b, v), b, v);
    for (auto& b : basis) axpy(-dot(b, v), b, v);
    const double nv = norm2(v);
    if (!(nv > 1e-14 * (norm2(u) + 1e-300))) return;
    for (auto& e : v) e /= nv;
    basis.push_back(v);
    if ((int)basis.size() > warmMax) basis.erase(basis.begin());
  }

  static double pcgRate(const PcgResult& r) { return r.iters / std::max(std::log10(r.iters0 / std::max(r.relres, 1e-300)), 0.5); }

  // _pcg :1001-1042
  PcgResult pcg(const dvec& b, dvec& xv, double tl, int mit, double perDecade) {
    const Pattern& P = model->pattern; const double* val = model->val.data(); const size_t n = model->ndof;
    const auto& isC = model->isConstrained;
    fullMatVec(P, val, xv.data(), r.data());
    for (size_t i = 0; i < n; i++) r[i] = b[i] - r[i];
    if (!isC.empty()) for (size_t i = 0; i < n; i++) if (isC[i]) { r[i] = 0; xv[i] = 0; }
    const double bnorm = norm2(b);
    double rnorm = norm2(r);
    const double r0 = rnorm / bnorm;
    PcgResult out;
    if (rnorm / bnorm < tl) { out.iters = 0; out.relres = rnorm / bnorm; out.converged = true; out.iters0 = r0; return out; }
    if (perDecade > 0) mit = std::min(mit, std::max(REBUILD_MIN_ITERS, (int)std::ceil(perDecade * std::log10(r0 / tl))));
    pc->apply(r.data(), z.data());
    if (!isC.empty()) for (size_t i = 0; i < n; i++) if (isC[i]) z[i] = 0;
    p = z;
    double rz = dot(r, z);
    int it = 0;
    for (it = 1; it <= mit; it++) {
      fullMatVec(P, val, p.data(), q.data());
      const double pq = dot(p, q);
      if (!(pq > 0)) break;
      const double alpha = rz / pq;
      axpy(alpha, p, xv);
      axpy(-alpha, q, r);
      rnorm = norm2(r);
      if (rnorm / bnorm < tl) { out.iters = it; out.relres = rnorm / bnorm; out.converged = true; out.iters0 = r0; return out; }
      pc->apply(r.data(), z.data());
      if (!isC.empty()) for (size_t i = 0; i < n; i++) if (isC[i]) z[i] = 0;
      const double rz2 = dot(r, z);
      const double beta = rz2 / rz;
      rz = rz2;
      for (size_t i = 0; i < n; i++) p[i] = z[i] + beta * p[i];
    }
    out.iters = std::min(it, mit); out.relres = rnorm / bnorm; out.converged = false; out.iters0 = r0;
    return out;
  }

  // solve :933-994; model values are scaled in place
  void solve(const double* f, double* u, long key, SolveInfo& info) {
    const double t0 = now_ms();
    const size_t n = model->ndof;
    if (key != -1 && key != pcKey) needRebuild = true;
    pcKey = key;
    scale();
    for (size_t qq = 0; qq < n; qq++) bs[qq] = f[qq] * s[qq];
    const double bnorm = norm2(bs);
    info = SolveInfo();
    if (bnorm == 0) {
      std::fill(u, u + n, 0.0);
      info.converged = 1; info.ms = now_ms() - t0; info.precond = pcKind < 0 ? precondKind : pcKind; info.warm = (int)basis.size();
      return;
    }
    bool rebuilt = false; double pcMs = 0;
    if (!pc || needRebuild) { pcMs = buildPC(precondKind); rebuilt = true; }
    warmStart(bs, x);
    PcgResult res = pcg(bs, x, tol, maxit, rebuilt ? 0 : REBUILD_FACTOR * ratePerDecade);
    bool fallback = false; int totalIters = res.iters;
    if (!res.converged && !rebuilt) {
      pcMs += buildPC(precondKind); rebuilt = true;
      res = pcg(bs, x, tol, maxit, 0);
      totalIters += res.iters;
    }
    if (!res.converged) {
      const int other = pcKind == 0 ? 1 : 0;
      fallback = true;
      pcMs += buildPC(other); rebuilt = true;
      res = pcg(bs, x, tol, maxit, 0);
      totalIters += res.iters;
      needRebuild = true;
    }
    if (!fallback && res.converged) {
      const bool known = ratePerDecade > 0 && !rebuilt;
      if (known) { if (pcgRate(res) > REBUILD_FACTOR * ratePerDecade) needRebuild = true; }
      else ratePerDecade = std::log10(res.iters0 / std::max(res.relres, 1e-300)) >= 1 ? pcgRate(res) : 0;
    }
    res.iters = totalIters;
    dvec uu(n);
    for (size_t qq = 0; qq < n; qq++) uu[qq] = x[qq] * s[qq];
    if (res.converged) storeSolution(uu);
    std::copy(uu.begin(), uu.end(), u);
    info.iters = res.iters; info.relres = res.relres; info.converged = res.converged; info.iters0 = res.iters0;
    info.ms = now_ms() - t0; info.pcMs = pcMs; info.precond = pcKind; info.rebuilt = rebuilt; info.warm = (int)basis.size();
    info.fallback = fallback;
    if (auto* mg = dynamic_cast<MultigridPC*>(pc.get())) { info.colJitter = mg->colJitter; info.shellJitter = mg->shellJitter; info.levels = (int)mg->levels.size(); }
  }
};

// ---- Anand viscoplastic point (src/core/13-fatigue.js:13-237) --------------------------
struct AnandParams { double A, QR, xi, m, shat, n, h0, a, s0, nu; };

// gridAt (03-materials.js:347-355) on the 1 degC grid from TGRID_MIN
double gridAt(const double* arr, double T) {
  const double x = T - TGRID_MIN;
  if (x <= 0) return arr[0];
  if (x >= TGRID_N - 1) return arr[TGRID_N - 1];
  const int i = (int)std::floor(x); const double t = x - i;
  const double a = arr[i], b = arr[i + 1];
  return a + t * (b - a);
}

double sgn(double v) { return v > 0 ? 1 : (v < 0 ? -1 : 0); }

struct StepK { double G, K, expQ, rate0, dt; };

struct AnandPoint {
  AnandParams P;
  const double* Etab;
  double ep[6], s, ebar, W, sigEq, lastD;
  double tr_ep[6], tr_s, tr_ebar, tr_W, tr_sigEq, tr_dEbar;

  AnandPoint(const AnandParams& p, const double* E) : P(p), Etab(E) { reset(); }
  void reset() { for (auto& v : ep) v = 0; s = P.s0; ebar = 0; W = 0; sigEq = 0; lastD = 0; }

  // stepConstants :61-65
  StepK stepConstants(double T, double dt) const {
    const double E = gridAt(Etab, T), nu = P.nu;
    const double expQ = std::exp(P.QR / (T + KELVIN));
    return StepK{E / (2 * (1 + nu)), E / (3 * (1 - 2 * nu)), expQ, dt * P.A / expQ, dt};
  }

  // _solveS :32-52
  double solveS(double d, double dt, double expQ) const {
    if (d <= 0) return s;
    const double sstar = P.shat * std::pow(d / (dt * P.A) * expQ, P.n);
    const double sn = s, h0 = P.h0, a = P.a;
    auto phi = [&](double sv) { const double B = 1 - sv / sstar; return sv - sn - h0 * std::pow(std::fabs(B), a) * sgn(B) * d; };
    double lo = std::min(sn, sstar), hi = std::max(sn, sstar);
    if (hi - lo < 1e-14) return sn;
    double sv = 0.5 * (lo + hi);
    for (int it = 0; it < ANAND_NEWTON_MAXIT; it++) {
      const double f = phi(sv);
      if (std::fabs(f) < ANAND_TOL * std::max(1.0, sn)) break;
      if (f > 0) hi = sv; else lo = sv;
      const double B = 1 - sv / sstar;
      const double dphi = 1 + h0 * a * std::pow(std::fabs(B), a - 1) * d / sstar;
      double sn1 = sv - f / dphi;
      if (!(sn1 > lo && sn1 < hi)) sn1 = 0.5 * (lo + hi);
      if (std::fabs(sn1 - sv) < 1e-15 * std::max(1.0, sv)) { sv = sn1; break; }
      sv = sn1;
    }
    return sv;
  }

  // _dsdd :209-218
  double dsdd(double d, double sv, double dt, double expQ) const {
    if (d <= 0) return 0;
    const double sstar = P.shat * std::pow(d / (dt * P.A) * expQ, P.n);
    const double B = 1 - sv / sstar;
    const double absB = std::fabs(B), sg = sgn(B);
    const double h0 = P.h0, a = P.a, n = P.n;
    const double dphi_ds = 1 + h0 * a * std::pow(absB, a - 1) * d / sstar;
    const double dphi_dd = -h0 * std::pow(absB, a) * sg - h0 * a * std::pow(absB, a - 1) * sv * n / sstar;
    return -dphi_dd / dphi_ds;
  }

  // step :67-143
  double step(const double* eps, double T, double dt, double* sig, double* D, bool wantTangent, const StepK* kin) {
    const StepK k = kin ? *kin : stepConstants(T, dt);
    const double G = k.G, K = k.K, expQ = k.expQ, rate0 = k.rate0;
    const double vol = (eps[0] + eps[1] + eps[2]) / 3;
    double e[6], str[6], nvec[6];
    e[0] = eps[0] - vol - ep[0]; e[1] = eps[1] - vol - ep[1]; e[2] = eps[2] - vol - ep[2];
    e[3] = 0.5 * eps[3] - ep[3]; e[4] = 0.5 * eps[4] - ep[4]; e[5] = 0.5 * eps[5] - ep[5];
    for (int i = 0; i < 6; i++) str[i] = 2 * G * e[i];
    const double nrm = std::sqrt(str[0] * str[0] + str[1] * str[1] + str[2] * str[2] + 2 * (str[3] * str[3] + str[4] * str[4] + str[5] * str[5]));
    const double sigTr = std::sqrt(1.5) * nrm;
    double d = 0, s1 = s, dDdSig = 0;
    if (sigTr > 1e-14 && dt > 0) {
      const double dmax = sigTr / (3 * G);
      struct G_ { double g, s, x, sh; };
      auto gfun = [&](double dd) {
        const double sv = solveS(dd, dt, expQ);
        const double x = P.xi * (sigTr - 3 * G * dd) / sv;
        const double sh = std::sinh(x);
        return G_{dd - rate0 * std::pow(sh, 1 / P.m), sv, x, sh};
      };
      double lo = 0, hi = dmax;
      double dd = lastD > 0 && lastD < dmax ? lastD : std::min(dmax, rate0 * std::pow(std::sinh(P.xi * sigTr / s), 1 / P.m));
      if (!std::isfinite(dd) || dd <= 0) dd = 0.5 * dmax;
      G_ res{0, s, 0, 0};
      for (int it = 0; it < ANAND_NEWTON_MAXIT; it++) {
        res = gfun(dd);
        if (!std::isfinite(res.g)) { lo = dd; dd = 0.5 * (lo + hi); continue; }
        if (std::fabs(res.g) < ANAND_TOL * std::max(dmax, 1e-30)) break;
        if (res.g > 0) hi = dd; else lo = dd;
        const double fx = rate0 * (1 / P.m) * std::pow(res.sh, 1 / P.m - 1) * std::cosh(res.x);
        const double ds = dsdd(dd, res.s, dt, expQ);
        const double sg = sigTr - 3 * G * dd;
        const double dg = 1 + fx * P.xi * (3 * G / res.s + sg * ds / (res.s * res.s));
        double dn = dd - res.g / dg;
        if (!(dn > lo && dn < hi) || !std::isfinite(dn)) dn = 0.5 * (lo + hi);
        if (std::fabs(dn - dd) < 1e-16 * std::max(dmax, 1e-30)) { dd = dn; break; }
        dd = dn;
      }
      d = dd; s1 = res.s;
      lastD = d;
      if (wantTangent) {
        const double fx = rate0 * (1 / P.m) * std::pow(res.sh, 1 / P.m - 1) * std::cosh(res.x);
        const double ds = dsdd(dd, res.s, dt, expQ);
        const double sg = sigTr - 3 * G * dd;
        const double dg = 1 + fx * P.xi * (3 * G / res.s + sg * ds / (res.s * res.s));
        dDdSig = (fx * P.xi / res.s) / dg;
      }
    }
    const double theta = sigTr > 1e-14 ? 1 - 3 * G * d / sigTr : 1;
    if (nrm > 0) for (int i = 0; i < 6; i++) nvec[i] = str[i] / nrm; else for (int i = 0; i < 6; i++) nvec[i] = 0;
    const double dg = std::sqrt(1.5) * d;
    for (int i = 0; i < 6; i++) tr_ep[i] = ep[i] + dg * nvec[i];
    const double sm = 3 * K * vol;
    sig[0] = theta * str[0] + sm; sig[1] = theta * str[1] + sm; sig[2] = theta * str[2] + sm;
    sig[3] = theta * str[3]; sig[4] = theta * str[4]; sig[5] = theta * str[5];
    const double sEq = sigTr - 3 * G * d;
    tr_s = s1; tr_ebar = ebar + d; tr_W = W + 0.5 * (sigEq + sEq) * d; tr_sigEq = sEq; tr_dEbar = d;
    if (wantTangent) {
      const double thetaBar = 2 * G * 1.5 * dDdSig - (1 - theta);
      const double c1 = 2 * G * theta, c2 = 2 * G * thetaBar;
      for (int i = 0; i < 6; i++) for (int j = 0; j < 6; j++) {
        double v = -c2 * nvec[i] * nvec[j];
        if (i < 3 && j < 3) v += K + c1 * ((i == j ? 1 : 0) - 1.0 / 3);
        else if (i == j) v += 0.5 * c1;
        D[i * 6 + j] = v;
      }
    }
    return d;
  }

  // stepColumn :153-166
  double stepColumn(double* eps, double T, double dt, double* sig, double* D, const StepK* k) {
    const int Pi[3] = {0, 1, 3};
    double A[9], Ai[9];
    double d = 0;
    for (int it = 0; it < COLUMN_NEWTON_MAXIT; it++) {
      d = step(eps, T, dt, sig, D, true, k);
      const double r0 = sig[0], r1 = sig[1], r2 = sig[3];
      const double ref = std::max(std::max(1.0, std::fabs(sig[2])), std::max(std::fabs(sig[4]), std::fabs(sig[5])));
      if (std::max(std::max(std::fabs(r0), std::fabs(r1)), std::fabs(r2)) < COLUMN_STRESS_TOL * ref) break;
      for (int r = 0; r < 3; r++) for (int c = 0; c < 3; c++) A[3 * r + c] = D[6 * Pi[r] + Pi[c]];
      inv3(A, Ai);
      for (int r = 0; r < 3; r++) eps[Pi[r]] -= Ai[3 * r] * r0 + Ai[3 * r + 1] * r1 + Ai[3 * r + 2] * r2;
    }
    return d;
  }

  // stepSeriesColumn :178-206: the solder cap (height fraction fs) in series with an elastic
  // pillar of compliances Cp; tz = prescribed column-average (zz, yz, zx) mechanical strains
  double stepSeriesColumn(double* eps, const double* tz, double fs, const double* Cp, double T, double dt, double* sig, double* D,
                          const StepK* k) {
    const int Pi[3] = {0, 1, 3}, Z[3] = {2, 4, 5}, ord[6] = {0, 1, 3, 2, 4, 5};
    const double fp = 1 - fs;
    double J[36], R[6];
    const double E = gridAt(Etab, T);
    double d = 0;
    for (int it = 0; it < COLUMN_NEWTON_MAXIT; it++) {
      d = step(eps, T, dt, sig, D, true, k);
      for (int r = 0; r < 3; r++) { R[r] = sig[Pi[r]]; R[3 + r] = fs * eps[Z[r]] + fp * Cp[r] * sig[Z[r]] - tz[r]; }
      const double ref = std::max(std::max(1.0, std::fabs(sig[2])), std::max(std::fabs(sig[4]), std::fabs(sig[5])));
      double worst = 0;
      for (int r = 0; r < 3; r++) worst = std::max(std::max(worst, std::fabs(R[r])), std::fabs(R[3 + r]) * E);
      if (worst < COLUMN_STRESS_TOL * ref) break;
      for (int r = 0; r < 6; r++)
        for (int c = 0; c < 6; c++) {
          const double Dv = D[6 * ord[r] + ord[c]];
          J[6 * r + c] = r < 3 ? Dv : fp * Cp[r - 3] * Dv + (ord[r] == ord[c] ? fs : 0);
        }
      // Gaussian elimination with partial pivoting
      for (int c = 0; c < 6; c++) {
        int pr = c;
        for (int r = c + 1; r < 6; r++) if (std::fabs(J[6 * r + c]) > std::fabs(J[6 * pr + c])) pr = r;
        if (pr != c) {
          for (int q = 0; q < 6; q++) std::swap(J[6 * c + q], J[6 * pr + q]);
          std::swap(R[c], R[pr]);
        }
        const double piv = J[7 * c];
        for (int r = c + 1; r < 6; r++) {
          const double f = J[6 * r + c] / piv;
          if (f == 0) continue;
          for (int q = c; q < 6; q++) J[6 * r + q] -= f * J[6 * c + q];
          R[r] -= f * R[c];
        }
      }
      for (int c = 5; c >= 0; c--) {
        double v = R[c];
        for (int q = c + 1; q < 6; q++) v -= J[6 * c + q] * R[q];
        R[c] = v / J[7 * c];
      }
      for (int c = 0; c < 6; c++) eps[ord[c]] -= R[c];
    }
    return d;
  }

  void commit() { for (int i = 0; i < 6; i++) ep[i] = tr_ep[i]; s = tr_s; ebar = tr_ebar; W = tr_W; sigEq = tr_sigEq; }
};


// ---- bump submodel (BumpSubmodel, 13-fatigue.js:470-1104) ----------------------------------------
const double SUB_T_AVG = 0.025;             // 00-constants.js:114
const int SUB_NEWTON_MAXIT = 25;            // :116
const double SUB_RES_TOL = 1e-6, SUB_DU_TOL = 1e-8, SUB_INNER_TOL = 1e-8;   // :117-119
const double INELASTIC_STEP_MAX = 2e-4;     // :113

// gridAt with stride and component (03-materials.js:347-355)
double gridAtS(const double* arr, double T, int stride, int comp) {
  const double x = T - TGRID_MIN;
  if (x <= 0) return arr[comp];
  if (x >= TGRID_N - 1) return arr[(TGRID_N - 1) * stride + comp];
  const int i = (int)std::floor(x); const double t = x - i;
  const double a = arr[i * stride + comp], b = arr[(i + 1) * stride + comp];
  return a + t * (b - a);
}

// gridAddAt (03-materials.js:358-362)
void gridAddAt(const double* grid, double T, int stride, int n, double w, double* out) {
  double x = T - TGRID_MIN;
  x = x < 0 ? 0 : (x > TGRID_N - 1 ? TGRID_N - 1 : x);
  const int i = std::min((int)std::floor(x), TGRID_N - 2); const double t = x - i;
  const int a = i * stride, b = a + stride;
  for (int c = 0; c < n; c++) out[c] += w * (grid[a + c] + t * (grid[b + c] - grid[a + c]));
}

// forGridSegments (03-materials.js:370-377)
template <class F> void forGridSegments(double Ta, double Tb, F fn) {
  const double lo = std::min(Ta, Tb), hi = std::max(Ta, Tb);
  for (double t0 = lo; t0 < hi - 1e-12;) {
    const double t1 = std::min(hi, TGRID_MIN + std::floor(t0 - TGRID_MIN + 1e-9) + 1);
    fn(0.5 * (t0 + t1), t0, t1);
    t0 = t1;
  }
}

// gridMean (03-materials.js:380-387)
void gridMean(const double* grid, int stride, int n, double Ta, double Tb, double* out) {
  for (int c = 0; c < n; c++) out[c] = 0;
  const double L = std::fabs(Tb - Ta);
  if (L < 1e-12) { gridAddAt(grid, Ta, stride, n, 1, out); return; }
  forGridSegments(Ta, Tb, [&](double tm, double t0, double t1) { gridAddAt(grid, tm, stride, n, (t1 - t0) / L, out); });
}

// gridStressIncrement with a stiffness grid (03-materials.js:394-410)
void gridStressIncrement(const double* Dg, const double* Fg, double Ta, double Tb, double* out) {
  for (int r = 0; r < 6; r++) out[r] = 0;
  const double sg = Tb >= Ta ? 1 : -1;
  double D[36];
  forGridSegments(Ta, Tb, [&](double tm, double t0, double t1) {
    for (auto& v : D) v = 0;
    gridAddAt(Dg, tm, 36, 36, 1, D);
    const double f0 = gridAtS(Fg, t1, 3, 0) - gridAtS(Fg, t0, 3, 0), f1 = gridAtS(Fg, t1, 3, 1) - gridAtS(Fg, t0, 3, 1),
                 f2 = gridAtS(Fg, t1, 3, 2) - gridAtS(Fg, t0, 3, 2);
    for (int r = 0; r < 6; r++) out[r] += sg * (D[6 * r] * f0 + D[6 * r + 1] * f1 + D[6 * r + 2] * f2);
  });
}

// gridModulusStrainIncrement (03-materials.js:413-418)
double gridModulusStrainIncrement(const double* E, const double* F, double Ta, double Tb) {
  const double sg = Tb >= Ta ? 1 : -1;
  double s = 0;
  forGridSegments(Ta, Tb, [&](double tm, double t0, double t1) { s += gridAt(E, tm) * (gridAt(F, t1) - gridAt(F, t0)); });
  return sg * s;
}

// isoD through isoEC and orthoD (03-materials.js:222-249)
void isoD(double E, double nu, double nuMax, double* out) {
  const double nc = std::min(nu, nuMax);
  const double G = E / (2 * (1 + nc));
  const double nxy = std::min(nc, nuMax), nxz = nxy, nyz = nxy;
  double S[9] = {0}, C[9] = {0};
  S[0] = 1 / E; S[4] = 1 / E; S[8] = 1 / E;
  S[1] = S[3] = -nxy / E;
  S[2] = S[6] = -nxz / E;
  S[5] = S[7] = -nyz / E;
  invDense(S, 3, C);
  for (int q = 0; q < 36; q++) out[q] = 0;
  out[0] = C[0]; out[1] = C[1]; out[2] = C[2];
  out[6] = C[3]; out[7] = C[4]; out[8] = C[5];
  out[12] = C[6]; out[13] = C[7]; out[14] = C[8];
  out[21] = G; out[28] = G; out[35] = G;
}

// bbarMatrix (13-fatigue.js:474-491): B-bar (mean dilatation) matrix of a box element at a point
void bbarMatrix(double hx, double hy, double hz, double xi, double eta, double zeta, double* Bb) {
  double dx[11], dy[11], dz[11], cx[11], cy[11], cz[11];
  boxDerivs(hx, hy, hz, xi, eta, zeta, dx, dy, dz);
  boxDerivs(hx, hy, hz, 0, 0, 0, cx, cy, cz);
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

int findIntervalV(const dvec& a, double x) {
  const int n = (int)a.size();
  if (x <= a[0]) return 0;
  if (x >= a[n - 1]) return n - 2;
  int lo = 0, hi = n - 1;
  while (hi - lo > 1) { const int mid = (lo + hi) >> 1; if (a[mid] <= x) lo = mid; else hi = mid; }
  return lo;
}

// Inputs of a submodel: the voxel cell (materials per cell: 0 substrate slice, 1 solder,
// 2 underfill, 3 silicon), the global fields it is cut from (at the global temperatures ts, only
// the nglob global nodes the boundary uses, plus the 25 degC field) with every boundary node's 8
// global nodes and trilinear weights, and the material tables on the 1 degC grid.
struct SubInput {
  int nx, ny, nz; dvec xs, ys, zs; ivec cellMat;
  int nglob, nt; dvec ts, fields, u25; ivec bGlob; dvec bW;
  AnandParams anand; dvec solderE, solderF; int elasticSolder = 0;
  dvec ufE, ufF; double ufNu = 0.35;
  dvec siD, siF; dvec subD, subF;
  double nuMax = 0.49, zt = 0, zaf = 0;
  // homogenized-layer consistency mode (opts.uniformMaterial, 13-fatigue.js:516, 538, 556,
  // 711-748, 757): solder volume fraction of the bump layer (die.density), the global Poisson
  // clamp, and the top substrate band's section (buildBandSection, 04-homogenize.js:139-183):
  // per sub-layer its z range, shell stiffness table (36 x TGRID_N) and thermal strain table
  // (3 x TGRID_N)
  int uniform = 0; double density = 0, nuMaxGlobal = 0.45;
  int nsec = 0; dvec secZ, secD, secF;
};

// columnD (03-materials.js:259-266): the solder phase as separate columns, in-plane terms at
// COLUMN_INPLANE_FRACTION (00-constants.js:25) of the axial ones
void columnD(double E, double nu, double* out) {
  const double fl = 1e-3, G = E / (2 * (1 + nu));
  for (int q = 0; q < 36; q++) out[q] = 0;
  out[0] = out[7] = fl * E; out[21] = fl * G;
  out[14] = E; out[28] = G; out[35] = G;
}

struct Submodel {
  enum { SUB = 0, SOLDER = 1, UF = 2, SI = 3 };
  SubInput in;
  Mesh m;
  Pattern P;
  int ndof = 0;
  ivec bmap, eBb;
  std::vector<dvec> bbB; dvec bbW;
  std::vector<char> isC;
  ivec bNodes;
  std::vector<std::unique_ptr<AnandPoint>> anand;
  dvec u, uN, sigE, eFn, eK, eF, val, vals, s_;
  double Tn = 25;
  bool haveStepKey = false; double keyTn = 0, keyT = 0;
  // step records of the elastic materials: 4 materials, then (consistency mode) one per
  // substrate element layer
  std::vector<char> elasValid; dvec elasD, elasS;
  std::unique_ptr<ICPC> pc; bool pcStale = false; int pcIters = 0;

  explicit Submodel(const SubInput& inp) : in(inp) {
    m.nx = in.nx; m.ny = in.ny; m.nz = in.nz; m.xs = in.xs; m.ys = in.ys; m.zs = in.zs;
    const int ncells = (in.nx - 1) * (in.ny - 1) * (in.nz - 1);
    // consistency mode: the bump layer's phases are one homogenized material (13-fatigue.js:538)
    if (in.uniform)
      for (int& c : in.cellMat)
        if (c == SOLDER) c = UF;
    ivec cg(2 * ncells, -1), cp(2 * ncells, 0); dvec cs(2 * ncells, 0.0);
    for (int c = 0; c < ncells; c++) { cg[2 * c] = in.cellMat[c]; cp[2 * c] = in.cellMat[c]; cs[2 * c] = 1; }
    buildStructuredMesh(m, cg.data(), cp.data(), cs.data());
    ndof = 3 * m.nn;
    P = fullPatternFromUpper(bcsrFromElements(m.nn, m.conn, m.ne, 8));
    val.assign((size_t)P.nb * 9, 0.0);
    // _blockMap (13-fatigue.js:597-608)
    bmap.assign((size_t)m.ne * 64, -1);
    for (int e = 0; e < m.ne; e++) for (int a = 0; a < 8; a++) {
      const int na = m.conn[8 * e + a];
      for (int b = 0; b < 8; b++) {
        const int nb = m.conn[8 * e + b];
        int lo = P.rowPtr[na], hi = P.rowPtr[na + 1] - 1, k = -1;
        while (lo <= hi) { const int mid = (lo + hi) >> 1; const int v = P.col[mid]; if (v == nb) { k = mid; break; } if (v < nb) lo = mid + 1; else hi = mid - 1; }
        bmap[((size_t)e * 8 + a) * 8 + b] = k;
      }
    }
    // Gauss-point material states
    for (int e = 0; e < m.ne; e++) for (int g = 0; g < 8; g++)
      anand.emplace_back(m.eGroup[e] == SOLDER && !in.elasticSolder ? new AnandPoint(in.anand, in.solderE.data()) : nullptr);
    // _boundary: nodes on the six faces of the cell, in node order
    isC.assign(ndof, 0);
    std::vector<char> isB(m.nn, 0);
    for (int i = 0; i < m.nx; i++) for (int j = 0; j < m.ny; j++) for (int k = 0; k < m.nz; k++) {
      const int n = m.nodeId[((size_t)i * m.ny + j) * m.nz + k];
      if (n >= 0 && (i == 0 || j == 0 || k == 0 || i == m.nx - 1 || j == m.ny - 1 || k == m.nz - 1)) isB[n] = 1;
    }
    for (int n = 0; n < m.nn; n++) if (isB[n]) { bNodes.push_back(n); isC[3 * n] = isC[3 * n + 1] = isC[3 * n + 2] = 1; }
    // _bbarCache: B-bar matrices of the 8 Gauss points per distinct element size (12 digits)
    std::map<std::string, int> keys;
    eBb.assign(m.ne, 0);
    const double GP = 1 / std::sqrt(3.0);
    for (int e = 0; e < m.ne; e++) {
      const int i = m.eIJK[3 * e], j = m.eIJK[3 * e + 1], k = m.eIJK[3 * e + 2];
      const double hx = m.xs[i + 1] - m.xs[i], hy = m.ys[j + 1] - m.ys[j], hz = m.zs[k + 1] - m.zs[k];
      char buf[96];
      snprintf(buf, sizeof buf, "%.11e|%.11e|%.11e", hx, hy, hz);
      auto it = keys.find(buf);
      if (it == keys.end()) {
        const int idx = (int)bbB.size();
        keys.emplace(buf, idx);
        dvec B(8 * 144);
        for (int g = 0; g < 8; g++) bbarMatrix(hx, hy, hz, HEX_XI[g] * GP, HEX_ETA[g] * GP, HEX_ZETA[g] * GP, B.data() + 144 * g);
        bbB.push_back(B); bbW.push_back(hx * hy * hz / 8);
        eBb[e] = idx;
      } else eBb[e] = it->second;
    }
    const int nrec = 4 + (in.nz - 1);
    elasValid.assign(nrec, 0); elasD.assign(36 * (size_t)nrec, 0.0); elasS.assign(6 * (size_t)nrec, 0.0);
    u.assign(ndof, 0.0); uN.assign(ndof, 0.0);
    sigE.assign((size_t)m.ne * 48, 0.0); eFn.assign((size_t)m.ne * 24, 0.0);
    eK.assign((size_t)m.ne * 576, 0.0); eF.assign((size_t)m.ne * 24, 0.0);
  }

  // prescribe (13-fatigue.js:680-694) with Analysis.fieldAt (11-analysis.js:317-324)
  void prescribe(double T, dvec& uu) const {
    const int i = findIntervalV(in.ts, T);
    double t = (T - in.ts[i]) / (in.ts[i + 1] - in.ts[i]);
    t = t < 0 ? 0 : (t > 1 ? 1 : t);
    const size_t G = 3 * (size_t)in.nglob;
    const double* a = in.fields.data() + G * i; const double* b = a + G;
    for (size_t q = 0; q < bNodes.size(); q++) {
      const int n = bNodes[q];
      double ux = 0, uy = 0, uz = 0;
      for (int c = 0; c < 8; c++) {
        const int gn = in.bGlob[8 * q + c]; const double w = in.bW[8 * q + c];
        const double tx = a[3 * gn] + t * (b[3 * gn] - a[3 * gn]), ty = a[3 * gn + 1] + t * (b[3 * gn + 1] - a[3 * gn + 1]),
                     tz = a[3 * gn + 2] + t * (b[3 * gn + 2] - a[3 * gn + 2]);
        ux += w * (tx - in.u25[3 * gn]); uy += w * (ty - in.u25[3 * gn + 1]); uz += w * (tz - in.u25[3 * gn + 2]);
      }
      uu[3 * n] = ux; uu[3 * n + 1] = uy; uu[3 * n + 2] = uz;
    }
  }

  // _elastic (13-fatigue.js:702-757); subZ: the element layer's mid-height for the substrate
  // slice in the consistency mode
  void elastic(int mat, double Ta, double Tb, double* D, double* sth, double subZ = 0) const {
    auto rowSum = [&](int r) { return D[r * 6] + D[r * 6 + 1] + D[r * 6 + 2]; };
    auto rowSumOf = [](const double* Dx, int r) { return Dx[r * 6] + Dx[r * 6 + 1] + Dx[r * 6 + 2]; };
    if (in.uniform && mat == UF) {
      // solder columns (columnD) and underfill superposed with volume fractions fb, 1 - fb
      const double fb = in.density;
      double Es, Eu, Ds[36], Du[36];
      gridMean(in.solderE.data(), 1, 1, Ta, Tb, &Es);
      gridMean(in.ufE.data(), 1, 1, Ta, Tb, &Eu);
      columnD(Es, in.anand.nu, Ds);
      isoD(Eu, in.ufNu, in.nuMaxGlobal, Du);
      const double fs = gridModulusStrainIncrement(in.solderE.data(), in.solderF.data(), Ta, Tb) / Es;
      const double fu = gridModulusStrainIncrement(in.ufE.data(), in.ufF.data(), Ta, Tb) / Eu;
      for (int q = 0; q < 36; q++) D[q] = fb * Ds[q] + (1 - fb) * Du[q];
      for (int r = 0; r < 6; r++) sth[r] = fb * rowSumOf(Ds, r) * fs + (1 - fb) * rowSumOf(Du, r) * fu;
      return;
    }
    auto isoStep = [&](const dvec& E, const dvec& F, double nu) {
      double Em;
      gridMean(E.data(), 1, 1, Ta, Tb, &Em);
      const double ef = gridModulusStrainIncrement(E.data(), F.data(), Ta, Tb) / Em;
      isoD(Em, nu, in.nuMax, D);
      for (int r = 0; r < 6; r++) sth[r] = rowSum(r) * ef;
    };
    if (mat == SI) {
      for (int q = 0; q < 36; q++) D[q] = in.siD[q];
      const double f = gridAt(in.siF.data(), Tb) - gridAt(in.siF.data(), Ta);
      for (int r = 0; r < 6; r++) sth[r] = rowSum(r) * f;
      return;
    }
    if (mat == UF) { isoStep(in.ufE, in.ufF, in.ufNu); return; }
    if (mat == SOLDER) { isoStep(in.solderE, in.solderF, in.anand.nu); return; }
    if (in.uniform) {
      // the top band's own sub-layer stiffness at this height, with the through-thickness
      // response of the whole band: Voigt thickness modulus and Turner-weighted thermal strain
      const size_t DN = 36 * (size_t)TGRID_N, FN = 3 * (size_t)TGRID_N;
      int sl = in.nsec - 1;
      for (int q = 0; q < in.nsec; q++)
        if (subZ <= in.secZ[2 * q + 1] + 1e-12) { sl = q; break; }
      gridMean(in.secD.data() + DN * sl, 36, 36, Ta, Tb, D);
      const double* Fsl = in.secF.data() + FN * sl;
      double dF[3];
      for (int c = 0; c < 2; c++) dF[c] = gridAtS(Fsl, Tb, 3, c) - gridAtS(Fsl, Ta, 3, c);
      double Ez = 0, EzF = 0, tt = 0, Dq[36], sq[6];
      for (int q = 0; q < in.nsec; q++) {
        const double ts = in.secZ[2 * q + 1] - in.secZ[2 * q];
        gridMean(in.secD.data() + DN * q, 36, 36, Ta, Tb, Dq);
        const double* Fq = in.secF.data() + FN * q;
        const double fx = gridAtS(Fq, Tb, 3, 0) - gridAtS(Fq, Ta, 3, 0), fy = gridAtS(Fq, Tb, 3, 1) - gridAtS(Fq, Ta, 3, 1);
        gridStressIncrement(in.secD.data() + DN * q, Fq, Ta, Tb, sq);
        Ez += ts * Dq[14]; EzF += ts * (sq[2] - Dq[12] * fx - Dq[13] * fy); tt += ts;
      }
      D[14] = Ez / tt; dF[2] = EzF / Ez;
      for (int r = 0; r < 6; r++) sth[r] = D[r * 6] * dF[0] + D[r * 6 + 1] * dF[1] + D[r * 6 + 2] * dF[2];
      return;
    }
    gridMean(in.subD.data(), 36, 36, Ta, Tb, D);
    gridStressIncrement(in.subD.data(), in.subF.data(), Ta, Tb, sth);
  }

  // _elasRec (13-fatigue.js:760-773): per material (per substrate layer in the consistency
  // mode), cached for the step from Tn to T
  void elasRec(int e, double T, const double** D, const double** sth) {
    const int mat = m.eGroup[e], k = m.eIJK[3 * e + 2];
    const bool perLayer = in.uniform && mat == SUB;
    const int key = perLayer ? 4 + k : mat;
    if (!elasValid[key]) {
      elastic(mat, Tn, T, &elasD[36 * (size_t)key], &elasS[6 * (size_t)key], perLayer ? 0.5 * (m.zs[k] + m.zs[k + 1]) : 0);
      elasValid[key] = 1;
    }
    *D = &elasD[36 * (size_t)key]; *sth = &elasS[6 * (size_t)key];
  }

  // assemble (13-fatigue.js:776-853): tangent (wantK) and internal force at u; returns max dEbar
  double assemble(double T, double dt, const dvec& uu, dvec& rint, bool wantK) {
    if (wantK) std::fill(val.begin(), val.end(), 0.0);
    std::fill(rint.begin(), rint.end(), 0.0);
    const bool fresh = !(haveStepKey && keyTn == Tn && keyT == T);
    if (fresh) std::fill(elasValid.begin(), elasValid.end(), 0);
    AnandPoint kAn(in.anand, in.solderE.data());
    const StepK kc = kAn.stepConstants(T, dt);
    const double fSolder = gridAt(in.solderF.data(), T) - gridAt(in.solderF.data(), 25);
    double dMax = 0;
    double ue[24], Ke[576], fe[24], DB[144], eps[6], epsM[6], sig[6], Dg[36];
    for (int e = 0; e < m.ne; e++) {
      const double* Ball = bbB[eBb[e]].data(); const double w = bbW[eBb[e]];
      for (int a = 0; a < 8; a++) { const int n = m.conn[8 * e + a]; ue[3 * a] = uu[3 * n]; ue[3 * a + 1] = uu[3 * n + 1]; ue[3 * a + 2] = uu[3 * n + 2]; }
      std::fill(Ke, Ke + 576, 0.0); std::fill(fe, fe + 24, 0.0);
      if (!anand[(size_t)e * 8]) {
        double* Kc = eK.data() + 576 * (size_t)e; double* fc = eF.data() + 24 * (size_t)e;
        if (fresh) {
          const double *D, *sth;
          elasRec(e, T, &D, &sth);
          std::fill(Kc, Kc + 576, 0.0); std::fill(fc, fc + 24, 0.0);
          for (int g = 0; g < 8; g++) {
            const double* Bb = Ball + 144 * g;
            for (int c = 0; c < 24; c++) { double sum = 0; for (int r = 0; r < 6; r++) sum += Bb[r * 24 + c] * sth[r]; fc[c] += w * sum; }
            for (int r = 0; r < 6; r++) for (int c = 0; c < 24; c++) { double sum = 0; for (int t = 0; t < 6; t++) sum += D[r * 6 + t] * Bb[t * 24 + c]; DB[r * 24 + c] = sum; }
            for (int a = 0; a < 24; a++) for (int b = a; b < 24; b++) { double sum = 0; for (int r = 0; r < 6; r++) sum += Bb[r * 24 + a] * DB[r * 24 + b]; Kc[a * 24 + b] += w * sum; }
          }
          for (int a = 0; a < 24; a++) for (int b = 0; b < a; b++) Kc[a * 24 + b] = Kc[b * 24 + a];
        }
        for (int a = 0; a < 8; a++) { const int n = m.conn[8 * e + a]; ue[3 * a] -= uN[3 * n]; ue[3 * a + 1] -= uN[3 * n + 1]; ue[3 * a + 2] -= uN[3 * n + 2]; }
        for (int a = 0; a < 24; a++) { double sum = eFn[24 * (size_t)e + a] - fc[a]; for (int b = 0; b < 24; b++) sum += Kc[a * 24 + b] * ue[b]; fe[a] = sum; }
        for (int a = 0; a < 8; a++) { const int n = m.conn[8 * e + a]; rint[3 * n] += fe[3 * a]; rint[3 * n + 1] += fe[3 * a + 1]; rint[3 * n + 2] += fe[3 * a + 2]; }
        if (wantK) for (int a = 0; a < 8; a++) for (int b = 0; b < 8; b++) {
          const size_t v = 9 * (size_t)bmap[((size_t)e * 8 + a) * 8 + b];
          for (int p = 0; p < 3; p++) for (int q = 0; q < 3; q++) val[v + 3 * p + q] += Kc[(3 * a + p) * 24 + 3 * b + q];
        }
        continue;
      }
      for (int g = 0; g < 8; g++) {
        const double* Bb = Ball + 144 * g;
        for (int r = 0; r < 6; r++) { double s = 0; for (int c = 0; c < 24; c++) s += Bb[r * 24 + c] * ue[c]; eps[r] = s; }
        AnandPoint& pt = *anand[(size_t)e * 8 + g];
        for (int r = 0; r < 6; r++) epsM[r] = eps[r];
        epsM[0] -= fSolder; epsM[1] -= fSolder; epsM[2] -= fSolder;
        const double d = pt.step(epsM, T, dt, sig, Dg, wantK, &kc);
        if (d > dMax) dMax = d;
        for (int c = 0; c < 24; c++) { double s = 0; for (int r = 0; r < 6; r++) s += Bb[r * 24 + c] * sig[r]; fe[c] += w * s; }
        if (wantK) {
          for (int r = 0; r < 6; r++) for (int c = 0; c < 24; c++) { double s = 0; for (int t = 0; t < 6; t++) s += Dg[r * 6 + t] * Bb[t * 24 + c]; DB[r * 24 + c] = s; }
          for (int a = 0; a < 24; a++) for (int b = a; b < 24; b++) { double s = 0; for (int r = 0; r < 6; r++) s += Bb[r * 24 + a] * DB[r * 24 + b]; Ke[a * 24 + b] += w * s; }
        }
      }
      for (int a = 0; a < 8; a++) { const int n = m.conn[8 * e + a]; rint[3 * n] += fe[3 * a]; rint[3 * n + 1] += fe[3 * a + 1]; rint[3 * n + 2] += fe[3 * a + 2]; }
      if (wantK) {
        for (int a = 0; a < 24; a++) for (int b = 0; b < a; b++) Ke[a * 24 + b] = Ke[b * 24 + a];
        for (int a = 0; a < 8; a++) for (int b = 0; b < 8; b++) {
          const size_t v = 9 * (size_t)bmap[((size_t)e * 8 + a) * 8 + b];
          for (int p = 0; p < 3; p++) for (int q = 0; q < 3; q++) val[v + 3 * p + q] += Ke[(3 * a + p) * 24 + 3 * b + q];
        }
      }
    }
    haveStepKey = true; keyTn = Tn; keyT = T;
    return dMax;
  }

  // _commitElastic (13-fatigue.js:856-872)
  void commitElastic(double T) {
    double due[24], de[6], sg[6];
    for (int e = 0; e < m.ne; e++) {
      if (anand[(size_t)e * 8]) continue;
      const double *D, *sth;
      elasRec(e, T, &D, &sth);
      const double* Ball = bbB[eBb[e]].data(); const double w = bbW[eBb[e]];
      for (int a = 0; a < 8; a++) { const int n = m.conn[8 * e + a]; for (int c = 0; c < 3; c++) due[3 * a + c] = u[3 * n + c] - uN[3 * n + c]; }
      double* fn = eFn.data() + 24 * (size_t)e;
      std::fill(fn, fn + 24, 0.0);
      for (int g = 0; g < 8; g++) {
        const double* Bb = Ball + 144 * g; double* so = sigE.data() + 48 * (size_t)e + 6 * g;
        for (int r = 0; r < 6; r++) { double s2 = 0; for (int c = 0; c < 24; c++) s2 += Bb[r * 24 + c] * due[c]; de[r] = s2; }
        for (int r = 0; r < 6; r++) { double s2 = -sth[r]; for (int c = 0; c < 6; c++) s2 += D[r * 6 + c] * de[c]; so[r] += s2; sg[r] = so[r]; }
        for (int c = 0; c < 24; c++) { double s2 = 0; for (int r = 0; r < 6; r++) s2 += Bb[r * 24 + c] * sg[r]; fn[c] += w * s2; }
      }
    }
    uN = u; Tn = T;
  }

  // _constrain (13-fatigue.js:874-883)
  void constrain() {
    for (int i = 0; i < P.n; i++) for (int k = P.rowPtr[i]; k < P.rowPtr[i + 1]; k++) {
      const int j = P.col[k];
      for (int p = 0; p < 3; p++) for (int q = 0; q < 3; q++) {
        const int r = 3 * i + p, c = 3 * j + q;
        if ((isC[r] || isC[c]) && r != c) val[9 * (size_t)k + 3 * p + q] = 0;
      }
    }
  }

  // _solve (13-fatigue.js:886-917): IC(0)-PCG on the Jacobi-scaled tangent
  int solve(const dvec& rhs, dvec& x, double tol) {
    const int n = ndof;
    vals = val;
    s_.assign(n, 0.0);
    for (int i = 0; i < P.n; i++) {
      const size_t v = 9 * (size_t)P.diag[i];
      s_[3 * i] = 1 / std::sqrt(std::max(vals[v], 1e-300)); s_[3 * i + 1] = 1 / std::sqrt(std::max(vals[v + 4], 1e-300));
      s_[3 * i + 2] = 1 / std::sqrt(std::max(vals[v + 8], 1e-300));
    }
    for (int i = 0; i < P.n; i++) for (int k = P.rowPtr[i]; k < P.rowPtr[i + 1]; k++) {
      const int j = P.col[k]; const size_t v = 9 * (size_t)k;
      for (int p = 0; p < 3; p++) for (int q = 0; q < 3; q++) vals[v + 3 * p + q] *= s_[3 * i + p] * s_[3 * j + q];
    }
    dvec b(n);
    for (int q = 0; q < n; q++) b[q] = rhs[q] * s_[q];
    if (!pc || pcStale) { pc.reset(new ICPC(P, vals)); pcStale = false; pcIters = 0; }
    dvec r(n), z(n), p(n), qv(n);
    std::fill(x.begin(), x.end(), 0.0);
    r = b;
    const double bn = norm2(b);
    if (bn == 0) return 0;
    pc->apply(r.data(), z.data()); p = z;
    double rz = dot(r, z);
    int it;
    for (it = 1; it <= 2000; it++) {
      fullMatVec(P, vals.data(), p.data(), qv.data());
      const double alpha = rz / dot(p, qv);
      axpy(alpha, p, x); axpy(-alpha, qv, r);
      if (norm2(r) / bn < tol) break;
      pc->apply(r.data(), z.data());
      const double rz2 = dot(r, z); const double beta = rz2 / rz; rz = rz2;
      for (int i = 0; i < n; i++) p[i] = z[i] + beta * p[i];
    }
    for (int q = 0; q < n; q++) x[q] *= s_[q];
    if (!pcIters) pcIters = it; else if (it > 2 * pcIters) pcStale = true;
    return it;
  }

  // stepTo (13-fatigue.js:924-956)
  bool stepTo(double T, double dt, int* newton, double* dMaxOut) {
    const int n = ndof;
    dvec rint(n), du(n), rhs(n);
    prescribe(T, u);
    double dMax = 0, rPrev = INFINITY;
    bool converged = false, haveK = false;
    int it;
    for (it = 1; it <= SUB_NEWTON_MAXIT; it++) {
      const bool wantK = it <= 2 || !haveK;
      dMax = assemble(T, dt, u, rint, wantK);
      if (wantK) { constrain(); haveK = true; }
      double rn = 0, fn = 0;
      for (int q = 0; q < n; q++) { if (!isC[q]) rn += rint[q] * rint[q]; fn += rint[q] * rint[q]; }
      rn = std::sqrt(rn); fn = std::sqrt(fn);
      const double ref = std::max(fn, 1e-30);
      if (rn / ref < SUB_RES_TOL) { converged = true; break; }
      if (!wantK && rn > 0.5 * rPrev) { assemble(T, dt, u, rint, true); constrain(); }
      rPrev = rn;
      for (int q = 0; q < n; q++) rhs[q] = isC[q] ? 0 : -rint[q];
      solve(rhs, du, std::max(SUB_INNER_TOL, std::min(1e-3, 0.01 * SUB_RES_TOL * ref / std::max(rn, 1e-300))));
      double dun = 0, un = 0;
      for (int q = 0; q < n; q++) { if (!isC[q]) { u[q] += du[q]; dun += du[q] * du[q]; } un += u[q] * u[q]; }
      if (std::sqrt(dun) < SUB_DU_TOL * std::max(std::sqrt(un), 1e-30)) { converged = true; it++; break; }
    }
    if (converged) {
      dMax = assemble(T, dt, u, rint, false);
      for (auto& pt : anand) if (pt) pt->commit();
      commitElastic(T);
    }
    *newton = it; *dMaxOut = dMax;
    return converged;
  }

  struct Snap { dvec u, sigE, eFn; double Tn; std::vector<std::array<double, 11>> st; };
  void snapshot(Snap& s) const {
    s.u = u; s.sigE = sigE; s.eFn = eFn; s.Tn = Tn;
    s.st.resize(anand.size());
    for (size_t i = 0; i < anand.size(); i++) if (anand[i]) {
      const AnandPoint& p = *anand[i];
      for (int c = 0; c < 6; c++) s.st[i][c] = p.ep[c];
      s.st[i][6] = p.s; s.st[i][7] = p.ebar; s.st[i][8] = p.W; s.st[i][9] = p.sigEq;
    }
  }
  void restore(const Snap& s) {
    u = s.u; uN = s.u; sigE = s.sigE; eFn = s.eFn; Tn = s.Tn;
    for (size_t i = 0; i < anand.size(); i++) if (anand[i]) {
      AnandPoint& p = *anand[i];
      for (int c = 0; c < 6; c++) p.ep[c] = s.st[i][c];
      p.s = s.st[i][6]; p.ebar = s.st[i][7]; p.W = s.st[i][8]; p.sigEq = s.st[i][9];
    }
  }

  // _stressSnapshot (13-fatigue.js:965-989): nodal stresses of every element (48: 8 nodes x 6,
  // float32) extrapolated from its Gauss points with GP_TO_NODE (07-element.js:227-234): the
  // committed Gauss-point stresses of elastic elements, and at solder points the stress of the
  // current displacement at the committed plastic strain (AnandPoint.stressAt, :221-227)
  void stressSnapshot(double T, float* out) const {
    double M[64];
    const double s3 = std::sqrt(3.0);
    for (int n = 0; n < 8; n++) {
      const double xi = HEX_XI[n] * s3, eta = HEX_ETA[n] * s3, zeta = HEX_ZETA[n] * s3;
      for (int g = 0; g < 8; g++) M[n * 8 + g] = 0.125 * (1 + HEX_XI[g] * xi) * (1 + HEX_ETA[g] * eta) * (1 + HEX_ZETA[g] * zeta);
    }
    double ue[24], eps[6], gp[48];
    for (int e = 0; e < m.ne; e++) {
      const double* Ball = bbB[eBb[e]].data();
      if (!anand[(size_t)e * 8]) {
        for (int q = 0; q < 48; q++) gp[q] = sigE[48 * (size_t)e + q];
      } else {
        for (int a = 0; a < 8; a++) { const int n = m.conn[8 * e + a]; ue[3 * a] = u[3 * n]; ue[3 * a + 1] = u[3 * n + 1]; ue[3 * a + 2] = u[3 * n + 2]; }
        for (int g = 0; g < 8; g++) {
          const double* Bb = Ball + 144 * g;
          for (int r = 0; r < 6; r++) { double sm = 0; for (int c = 0; c < 24; c++) sm += Bb[r * 24 + c] * ue[c]; eps[r] = sm; }
          const AnandPoint& pt = *anand[(size_t)e * 8 + g];
          const double f = gridAt(in.solderF.data(), T) - gridAt(in.solderF.data(), 25);
          eps[0] -= f; eps[1] -= f; eps[2] -= f;
          const double E = gridAt(in.solderE.data(), T), nu = in.anand.nu;
          const double G = E / (2 * (1 + nu)), K = E / (3 * (1 - 2 * nu));
          const double vol = (eps[0] + eps[1] + eps[2]) / 3, smv = 3 * K * vol;
          for (int i = 0; i < 3; i++) gp[6 * g + i] = 2 * G * (eps[i] - vol - pt.ep[i]) + smv;
          for (int i = 3; i < 6; i++) gp[6 * g + i] = 2 * G * (0.5 * eps[i] - pt.ep[i]);
        }
      }
      for (int a = 0; a < 8; a++)
        for (int c = 0; c < 6; c++) {
          double v = 0;
          for (int g = 0; g < 8; g++) v += M[a * 8 + g] * gp[6 * g + c];
          out[48 * (size_t)e + 6 * a + c] = (float)v;
        }
    }
  }

  // run (13-fatigue.js:1004-1104): the cycle history with adaptive sub-steps, the hysteresis
  // sampler of the two interface layers and the per-cycle inelastic work. out (10): dW, dWdie,
  // dWsub, dE, dEdie, dEsub, stabChange, steps, cutbacks, newtonPerStep; perCycle: dWdie, dWsub
  // per cycle; loop (4 per history point): tau, gamma (die side), tauSub, gammaSub. Stress
  // snapshots at the end of each ramp and dwell of the last cycle (:1053-1078): *nSnaps of them,
  // up to maxSnaps written, meta (4 each: T, t, cycle, phase) and 48 ne floats each.
  void run(int nsteps, const double* ht, const double* hT, const int* hcycle, const int* hphase, int cycles, double cphi, double sphi,
           double* out, double* perCycle, double* loop, int maxSnaps = 0, int* nSnaps = nullptr, double* snapMeta = nullptr,
           float* snapSig = nullptr) {
    if (nSnaps) *nSnaps = 0;
    struct Rec { int idx; double w; };
    std::vector<Rec> dieLayer, subLayer;
    for (int e = 0; e < m.ne; e++) {
      if (m.eGroup[e] != SOLDER) continue;
      const int k = m.eIJK[3 * e + 2]; const double zc = 0.5 * (m.zs[k] + m.zs[k + 1]);
      const int i = m.eIJK[3 * e], j = m.eIJK[3 * e + 1];
      const double w = (m.xs[i + 1] - m.xs[i]) * (m.ys[j + 1] - m.ys[j]) * (m.zs[k + 1] - m.zs[k]) / 8;
      for (int g = 0; g < 8; g++) {
        if (zc > in.zaf - SUB_T_AVG) dieLayer.push_back({e * 8 + g, w});
        if (zc < in.zt + SUB_T_AVG) subLayer.push_back({e * 8 + g, w});
      }
    }
    auto avg = [&](const std::vector<Rec>& list, bool W) {
      double sum = 0, ws = 0;
      for (const Rec& r : list) { sum += r.w * (W ? anand[r.idx]->W : anand[r.idx]->ebar); ws += r.w; }
      return ws ? sum / ws : NAN;
    };
    const double GP = 1 / std::sqrt(3.0);
    int sample = 0;
    auto sampleLoop = [&](double T) {
      double tS = 0, gS = 0, tB = 0, gB = 0, wS = 0, wB = 0;
      double Bb[144], ue[24], eps[6], sig[6], Dd[36];
      for (int li = 0; li < 2; li++) {
        for (const Rec& r : li == 0 ? dieLayer : subLayer) {
          const int e = r.idx / 8, g = r.idx % 8;
          const int i = m.eIJK[3 * e], j = m.eIJK[3 * e + 1], k = m.eIJK[3 * e + 2];
          bbarMatrix(m.xs[i + 1] - m.xs[i], m.ys[j + 1] - m.ys[j], m.zs[k + 1] - m.zs[k], HEX_XI[g] * GP, HEX_ETA[g] * GP, HEX_ZETA[g] * GP, Bb);
          for (int a = 0; a < 8; a++) { const int nn = m.conn[8 * e + a]; ue[3 * a] = u[3 * nn]; ue[3 * a + 1] = u[3 * nn + 1]; ue[3 * a + 2] = u[3 * nn + 2]; }
          for (int rr = 0; rr < 6; rr++) { double s2 = 0; for (int c = 0; c < 24; c++) s2 += Bb[rr * 24 + c] * ue[c]; eps[rr] = s2; }
          AnandPoint& pt = *anand[r.idx];
          const double f = gridAt(in.solderF.data(), T) - gridAt(in.solderF.data(), 25);
          eps[0] -= f; eps[1] -= f; eps[2] -= f;
          pt.step(eps, T, 1e-9, sig, Dd, false, nullptr);   // stress at the committed plastic state
          const double tau = sig[5] * cphi + sig[4] * sphi, gam = eps[5] * cphi + eps[4] * sphi;
          if (li == 0) { tS += r.w * tau; gS += r.w * gam; wS += r.w; } else { tB += r.w * tau; gB += r.w * gam; wB += r.w; }
        }
      }
      double* L = loop + 4 * (size_t)sample++;
      L[0] = wS ? tS / wS : NAN; L[1] = wS ? gS / wS : NAN; L[2] = wB ? tB / wB : NAN; L[3] = wB ? gB / wB : NAN;
    };
    dvec Wdie(cycles + 1, 0.0), Wsub(cycles + 1, 0.0), Edie(cycles + 1, 0.0), Esub(cycles + 1, 0.0);
    long long totalNewton = 0; int cutbacks = 0, steps = 0, nsubNext = 1;
    sampleLoop(25);
    for (int k = 1; k < nsteps; k++) {
      const double T0 = hT[k - 1], T1 = hT[k], t0s = ht[k - 1], t1s = ht[k];
      int nsub = nsubNext; bool done = false; double dLast = 0;
      for (int attempt = 0; attempt < 8 && !done; attempt++) {
        Snap snap;
        snapshot(snap);
        bool ok = true;
        for (int sI = 1; sI <= nsub; sI++) {
          const double T = T0 + (T1 - T0) * sI / nsub, dt = (t1s - t0s) / nsub;
          int newton; double dMax;
          const bool conv = stepTo(T, dt, &newton, &dMax);
          totalNewton += newton; steps++;
          dLast = dMax;
          if (!conv || dMax > INELASTIC_STEP_MAX) { ok = false; break; }
        }
        if (ok) done = true;
        else { restore(snap); nsub *= 2; cutbacks++; }
      }
      nsubNext = dLast > 0.5 * INELASTIC_STEP_MAX ? std::min(nsub * 2, 64) : (dLast < 0.2 * INELASTIC_STEP_MAX ? std::max(1, nsub >> 1) : nsub);
      if (!done) throw std::runtime_error("Submodel step failed to converge after cutbacks");
      sampleLoop(T1);
      const int c = hcycle[k];
      if (nSnaps && c == cycles && (k == nsteps - 1 || hphase[k + 1] != hphase[k])) {
        const int q = (*nSnaps)++;
        if (q < maxSnaps) {
          double* mt = snapMeta + 4 * (size_t)q;
          mt[0] = T1; mt[1] = t1s; mt[2] = c; mt[3] = hphase[k];
          stressSnapshot(T1, snapSig + 48 * (size_t)m.ne * q);
        }
      }
      Wdie[c] = avg(dieLayer, true); Wsub[c] = avg(subLayer, true);
      Edie[c] = avg(dieLayer, false); Esub[c] = avg(subLayer, false);
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
}  // namespace

// =====================================================================================
// C API for the test suite (ctypes) and the bench's CPU baseline leg
// =====================================================================================
extern "C" {

// ---- stress-history recovery and post-processing readers -------------------------------------

// findInterval (01-util.js:12-22)
int findIntervalD(const dvec& a, double x) {
  const int n = (int)a.size();
  if (x <= a[0]) return 0;
  if (x >= a[n - 1]) return n - 2;
  int lo = 0, hi = n - 1;
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (a[mid] <= x) lo = mid; else hi = mid;
  }
  return lo;
}

// boxStrainAt (07-element.js:127-142): engineering strain at (xi, eta, zeta) from the 24 nodal
// DOFs u and the 9 incompatible-mode amplitudes alpha
void boxStrainAt(double hx, double hy, double hz, const double* u, const double* alpha, double xi, double eta, double zeta, double* eps) {
  double dx[11], dy[11], dz[11];
  boxDerivs(hx, hy, hz, xi, eta, zeta, dx, dy, dz);
  for (int q = 0; q < 6; q++) eps[q] = 0;
  for (int b = 0; b < 11; b++) {
    const double ux = b < 8 ? u[3 * b] : alpha[3 * (b - 8)];
    const double uy = b < 8 ? u[3 * b + 1] : alpha[3 * (b - 8) + 1];
    const double uz = b < 8 ? u[3 * b + 2] : alpha[3 * (b - 8) + 2];
    eps[0] += dx[b] * ux; eps[1] += dy[b] * uy; eps[2] += dz[b] * uz;
    eps[3] += dy[b] * ux + dx[b] * uy;
    eps[4] += dz[b] * uy + dy[b] * uz;
    eps[5] += dz[b] * ux + dx[b] * uz;
  }
}

// cholSolveDense (01-util.js:94-107)
void cholSolveDense(const double* L, int n, double* b) {
  for (int i = 0; i < n; i++) {
    double s = b[i];
    const int ri = i * n;
    for (int k = 0; k < i; k++) s -= L[ri + k] * b[k];
    b[i] = s / L[ri + i];
  }
  for (int i = n - 1; i >= 0; i--) {
    double s = b[i];
    for (int k = i + 1; k < n; k++) s -= L[k * n + i] * b[k];
    b[i] = s / L[i * n + i];
  }
}

// The DOF increment of element e in the step assembled last (Model.accumulateStep,
// 09-assembly.js:508-528): du at its nodes, then the incompatible modes
// K_aa^-1 (f_a - K_au du) from the rows 24..32 of the step's shape matrices (stepRecovery
// :480-491) and, when the material is born, of the element thermal load
void elementIncrement(const Model& M, const double* du, int e, double* dq) {
  const Mesh& m = M.mesh;
  const PropSet& ps = M.psets[M.ePset[e]];
  const int i = m.eIJK[3 * e], j = m.eIJK[3 * e + 1], k = m.eIJK[3 * e + 2];
  const double hx = m.xs[i + 1] - m.xs[i], hy = m.ys[j + 1] - m.ys[j], hz = m.zs[k + 1] - m.zs[k];
  const double V8 = hx * hy * hz / 8;
  const double c[6] = {V8 * 4 / (hx * hx), V8 * 4 / (hy * hy), V8 * 4 / (hz * hz), V8 * 4 / (hx * hy), V8 * 4 / (hy * hz), V8 * 4 / (hz * hx)};
  double Kr[297], f33[33], Kaa[81], col[9];
  for (int r = 0; r < 297; r++) {
    const double* Ma = ps.M + 24 * 33 + r;
    Kr[r] = c[0] * Ma[0] + c[1] * Ma[1089] + c[2] * Ma[2178] + c[3] * Ma[3267] + c[4] * Ma[4356] + c[5] * Ma[5445];
  }
  std::fill(f33, f33 + 33, 0.0);
  if (ps.born) elementFth(hx, hy, hz, ps.layered ? ps.V : nullptr, ps.layered ? nullptr : ps.s0, f33);
  for (int a = 0; a < 8; a++) {
    const int n = m.conn[8 * e + a];
    dq[3 * a] = du[3 * n]; dq[3 * a + 1] = du[3 * n + 1]; dq[3 * a + 2] = du[3 * n + 2];
  }
  for (int r = 0; r < 9; r++) for (int t = 0; t < 9; t++) Kaa[r * 9 + t] = Kr[r * 33 + 24 + t];
  cholDense(Kaa, 9, 1e-14);
  for (int r = 0; r < 9; r++) {
    double s = f33[24 + r];
    for (int t = 0; t < 24; t++) s -= Kr[r * 33 + t] * dq[t];
    col[r] = s;
  }
  cholSolveDense(Kaa, 9, col);
  for (int r = 0; r < 9; r++) dq[24 + r] = col[r];
}

// Model.accumulateStep with qOnly (09-assembly.js:508-533): q (33) += the element's increment
void accumulateQ(const Model& M, const double* du, int e, double* q) {
  double dq[33];
  elementIncrement(M, du, e, dq);
  for (int r = 0; r < 33; r++) q[r] += dq[r];
}

const int STRAIN_MONO = 7;   // 09-assembly.js:168

// boxStrainPoly (09-assembly.js:176-196): strain of a box element as a polynomial in the natural
// coordinates, E (42) = six components per monomial 1, xi, eta, zeta, xi eta, eta zeta, xi zeta
void boxStrainPoly(double hx, double hy, double hz, const double* q, double* E) {
  for (int t = 0; t < 42; t++) E[t] = 0;
  const double sx = 2 / hx, sy = 2 / hy, sz = 2 / hz;
  for (int a = 0; a < 8; a++) {
    const double xa = HEX_XI[a], ya = HEX_ETA[a], za = HEX_ZETA[a], ux = q[3 * a], uy = q[3 * a + 1], uz = q[3 * a + 2];
    const double cx = xa * sx / 8, cy = ya * sy / 8, cz = za * sz / 8;
    const int mx[4] = {0, 2, 3, 5}, my[4] = {0, 1, 3, 6}, mz[4] = {0, 1, 2, 4};
    const double vx[4] = {cx, cx * ya, cx * za, cx * ya * za}, vy[4] = {cy, cy * xa, cy * za, cy * xa * za},
                 vz[4] = {cz, cz * xa, cz * ya, cz * xa * ya};
    for (int t = 0; t < 4; t++) { const int mm = mx[t]; const double cc = vx[t]; E[6 * mm] += cc * ux; E[6 * mm + 3] += cc * uy; E[6 * mm + 5] += cc * uz; }
    for (int t = 0; t < 4; t++) { const int mm = my[t]; const double cc = vy[t]; E[6 * mm + 1] += cc * uy; E[6 * mm + 3] += cc * ux; E[6 * mm + 4] += cc * uz; }
    for (int t = 0; t < 4; t++) { const int mm = mz[t]; const double cc = vz[t]; E[6 * mm + 2] += cc * uz; E[6 * mm + 4] += cc * uy; E[6 * mm + 5] += cc * ux; }
  }
  const double* a1 = q + 24; const double* a2 = q + 27; const double* a3 = q + 30;
  E[6 * 1] += -2 * sx * a1[0]; E[6 * 1 + 3] += -2 * sx * a1[1]; E[6 * 1 + 5] += -2 * sx * a1[2];
  E[6 * 2 + 1] += -2 * sy * a2[1]; E[6 * 2 + 3] += -2 * sy * a2[0]; E[6 * 2 + 4] += -2 * sy * a2[2];
  E[6 * 3 + 2] += -2 * sz * a3[2]; E[6 * 3 + 4] += -2 * sz * a3[1]; E[6 * 3 + 5] += -2 * sz * a3[0];
}

// Model.accumulateStep without qOnly (09-assembly.js:508-544): q += dq and, when the material is
// born, per sub-layer S_m += D_m E_m(dq) (m < 7) and S_th += the step's thermal stress increment
void accumulateState(const Model& M, const double* du, int e, double* state) {
  const Mesh& m = M.mesh;
  const PropSet& ps = M.psets[M.ePset[e]];
  double dq[33], E[42];
  elementIncrement(M, du, e, dq);
  for (int r = 0; r < 33; r++) state[r] += dq[r];
  if (!ps.born) return;
  const int i = m.eIJK[3 * e], j = m.eIJK[3 * e + 1], k = m.eIJK[3 * e + 2];
  boxStrainPoly(m.xs[i + 1] - m.xs[i], m.ys[j + 1] - m.ys[j], m.zs[k + 1] - m.zs[k], dq, E);
  const int ns = ps.layered ? ps.nsub : 1, blk = 6 * (STRAIN_MONO + 1);
  for (int s = 0; s < ns; s++) {
    const double* D = ps.layered ? ps.subD.data() + 36 * s : ps.D;
    const double* s0 = ps.layered ? ps.subS0.data() + 6 * s : ps.s0;
    const int o = 33 + s * blk;
    for (int mo = 0; mo < STRAIN_MONO; mo++) {
      for (int r = 0; r < 6; r++) { double v = 0; for (int t = 0; t < 6; t++) v += D[r * 6 + t] * E[6 * mo + t]; state[o + 6 * mo + r] += v; }
    }
    for (int r = 0; r < 6; r++) state[o + 6 * STRAIN_MONO + r] += s0[r];
  }
}

// stateStress (09-assembly.js:555-571) with subLayerAt (:547-552): total strain and stress of
// element e at the natural point nat from its history state
void stateStress(const Model& M, int e, const double* state, const double* nat, double* eps, double* sig) {
  const Mesh& m = M.mesh;
  const PropSet& ps = M.psets[M.ePset[e]];
  const int i = m.eIJK[3 * e], j = m.eIJK[3 * e + 1], k = m.eIJK[3 * e + 2];
  boxStrainAt(m.xs[i + 1] - m.xs[i], m.ys[j + 1] - m.ys[j], m.zs[k + 1] - m.zs[k], state, state + 24, nat[0], nat[1], nat[2], eps);
  int s = 0;
  if (ps.layered) {
    const double z = m.zs[k] + 0.5 * (nat[2] + 1) * (m.zs[k + 1] - m.zs[k]);
    s = ps.nsub - 1;
    for (int t = 0; t < ps.nsub; t++) if (z <= ps.subZ[2 * t + 1] + 1e-12) { s = t; break; }
  }
  const double phi[7] = {1, nat[0], nat[1], nat[2], nat[0] * nat[1], nat[1] * nat[2], nat[0] * nat[2]};
  const int o = 33 + s * 6 * (STRAIN_MONO + 1);
  for (int r = 0; r < 6; r++) {
    double v = -state[o + 6 * STRAIN_MONO + r];
    for (int mo = 0; mo < STRAIN_MONO; mo++) v += phi[mo] * state[o + 6 * mo + r];
    sig[r] = v;
  }
}

// boxStrainAt of element e (its dims from the mesh lines, Model.elementDims) with the element
// DOFs q at the natural point nat (siteStrainTable, 13-fatigue.js:335-342)
void elementStrain(const Model& M, int e, const double* q, const double* nat, double* eps) {
  const Mesh& m = M.mesh;
  const int i = m.eIJK[3 * e], j = m.eIJK[3 * e + 1], k = m.eIJK[3 * e + 2];
  boxStrainAt(m.xs[i + 1] - m.xs[i], m.ys[j + 1] - m.ys[j], m.zs[k + 1] - m.zs[k], q, q + 24, nat[0], nat[1], nat[2], eps);
}

// samplePlane (12-post.js:30-38) on plane k, component comp; NaN outside existing nodes
double samplePlane(const Mesh& m, const double* u, int k, int comp, double x, double y) {
  const int i = findIntervalD(m.xs, x), j = findIntervalD(m.ys, y);
  const double tx = (x - m.xs[i]) / (m.xs[i + 1] - m.xs[i]), ty = (y - m.ys[j]) / (m.ys[j + 1] - m.ys[j]);
  auto id = [&](int a, int b) { return m.nodeId[((size_t)(i + a) * m.ny + j + b) * m.nz + k]; };
  const int n00 = id(0, 0), n10 = id(1, 0), n01 = id(0, 1), n11 = id(1, 1);
  if (n00 < 0 || n10 < 0 || n01 < 0 || n11 < 0) return std::nan("");
  return (1 - tx) * (1 - ty) * u[3 * n00 + comp] + tx * (1 - ty) * u[3 * n10 + comp] + (1 - tx) * ty * u[3 * n01 + comp] +
         tx * ty * u[3 * n11 + comp];
}

// fitPlane (01-util.js:176-190)
void fitPlane(int n, const double* xs, const double* ys, const double* ws, double* c) {
  double sx = 0, sy = 0, sw = 0;
  for (int i = 0; i < n; i++) { sx += xs[i]; sy += ys[i]; sw += ws[i]; }
  const double mx = sx / n, my = sy / n, mw = sw / n;
  double sxx = 0, sxy = 0, syy = 0, sxw = 0, syw = 0;
  for (int i = 0; i < n; i++) {
    const double dx = xs[i] - mx, dy = ys[i] - my, dw = ws[i] - mw;
    sxx += dx * dx; sxy += dx * dy; syy += dy * dy; sxw += dx * dw; syw += dy * dw;
  }
  const double det = sxx * syy - sxy * sxy;
  double c1 = 0, c2 = 0;
  if (std::fabs(det) > 1e-300) { c1 = (sxw * syy - syw * sxy) / det; c2 = (syw * sxx - sxw * sxy) / det; }
  c[0] = mw - c1 * mx - c2 * my; c[1] = c1; c[2] = c2;
}

// warpageJEITA (12-post.js:60-109) without the shape class and the contour grid: signed
// magnitude, magnitude, sign, sign confidence and the fitted plane; out[7] = rmin, out[8] = rmax
void warpageJEITA(const Mesh& m, const double* u, int nb, const double* bx, const double* by, const double* zone, double* out) {
  const int DIAG_SAMPLES = 201;   // CONST.DIAG_SAMPLES (00-constants.js:98)
  auto sample = [&](double x, double y) { return samplePlane(m, u, 0, 2, x, y); };
  dvec w(nb), res(nb);
  for (int q = 0; q < nb; q++) w[q] = sample(bx[q], by[q]);
  double pl[3];
  fitPlane(nb, bx, by, w.data(), pl);
  double rmin = INFINITY, rmax = -INFINITY;
  for (int q = 0; q < nb; q++) {
    res[q] = w[q] - (pl[0] + pl[1] * bx[q] + pl[2] * by[q]);
    // Math.min / Math.max: NaN once any operand is NaN
    rmin = (std::isnan(res[q]) || std::isnan(rmin)) ? NAN : std::min(rmin, res[q]);
    rmax = (std::isnan(res[q]) || std::isnan(rmax)) ? NAN : std::max(rmax, res[q]);
  }
  const double mag = rmax - rmin;
  auto diag = [&](double xa, double ya, double xb, double yb, double& mx, double& mn) {
    const double wa = sample(xa, ya), wb = sample(xb, yb);
    mx = 0; mn = 0;
    for (int q = 0; q < DIAG_SAMPLES; q++) {
      const double t = (double)q / (DIAG_SAMPLES - 1);
      const double x = xa + t * (xb - xa), y = ya + t * (yb - ya);
      const double rel = sample(x, y) - (wa + t * (wb - wa));
      if (rel > mx) mx = rel;
      if (rel < mn) mn = rel;
    }
  };
  double abx, abn, cdx, cdn;
  diag(zone[0], zone[2], zone[1], zone[3], abx, abn);   // zone: x0, x1, y0, y1
  diag(zone[0], zone[3], zone[1], zone[2], cdx, cdn);
  const double sum = abx + abn + cdx + cdn;
  const double sign = sum > 0 ? 1 : (sum < 0 ? -1 : 0);
  out[0] = sign * mag; out[1] = mag; out[2] = sign; out[3] = mag > 0 ? std::fabs(sum) / mag : 0;
  out[4] = pl[0]; out[5] = pl[1]; out[6] = pl[2]; out[7] = rmin; out[8] = rmax;
}

struct orc_model { Model M; std::unique_ptr<LinearSolver> solver; std::string err; };

// cellGroup/cellPart/cellScale: two phases per cell (group < 0: none).
// ePsetOfGroup: property set of the elements of every homogeneous group; layered groups
// (groupLayered[g] = 1) take their property set per element layer k from secOfLayer[k].
// nconstr < 0 selects constraints321 with span `span`.
orc_model* orc_model_create(int nx, int ny, int nz, const double* xs, const double* ys, const double* zs,
                            const int* cellGroup, const int* cellPart, const double* cellScale,
                            int ngroups, const int* groupLayered, const int* groupStage, const int* groupPset,
                            const int* secOfLayer, int npset,
                            int nconstr, const int* constr, double span,
                            int nfx, const int* featureX, int nfy, const int* featureY) {
  auto* o = new orc_model();
  Model& M = o->M;
  Mesh& m = M.mesh;
  m.nx = nx; m.ny = ny; m.nz = nz;
  m.xs.assign(xs, xs + nx); m.ys.assign(ys, ys + ny); m.zs.assign(zs, zs + nz);
  buildStructuredMesh(m, cellGroup, cellPart, cellScale);
  if (nfx >= 0 && nfy >= 0 && (nfx > 0 || nfy > 0)) { m.featureX.assign(featureX, featureX + nfx); m.featureY.assign(featureY, featureY + nfy); m.hasFeatures = true; }
  M.ndof = 3 * m.nn;
  M.upper = bcsrFromElements(m.nn, m.conn, m.ne, 8);
  M.pattern = fullPatternFromUpper(M.upper);
  blockMap(M);
  M.val.assign((size_t)M.pattern.nb * 9, 0.0);
  M.groupStage.assign(groupStage, groupStage + ngroups);
  M.psets.resize(npset);
  M.ePset.assign(m.ne, 0);
  for (int e = 0; e < m.ne; e++) {
    const int g = m.eGroup[e];
    M.ePset[e] = groupLayered[g] ? secOfLayer[m.eIJK[3 * e + 2]] : groupPset[g];
  }
  if (nconstr < 0) M.constraints = constraints321(m, span);
  else M.constraints.assign(constr, constr + nconstr);
  o->solver.reset(new LinearSolver(&M));
  return o;
}

void orc_model_destroy(orc_model* o) { delete o; }

// the stacked modules' 3-2-1 support DOFs (mesh.moduleConstraints): the model's module constraints are
// the package's constraints followed by these (09-assembly.js:227)
void orc_set_module_constraints(orc_model* o, int n, const int* dofs) {
  Model& M = o->M;
  M.moduleConstraints = M.constraints;
  M.moduleConstraints.insert(M.moduleConstraints.end(), dofs, dofs + n);
  if (n <= 0) M.moduleConstraints.clear();
}

// sizes: nn, ne, nb, ndof, nconstr
void orc_model_sizes(orc_model* o, long* out) {
  out[0] = o->M.mesh.nn; out[1] = o->M.mesh.ne; out[2] = o->M.pattern.nb; out[3] = o->M.ndof; out[4] = (long)o->M.constraints.size();
}

void orc_model_mesh(orc_model* o, int* nodeId, int* conn, int* eIJK, int* colStart, int* cellElems, double* coords, int* constr, int* eGroup) {
  const Mesh& m = o->M.mesh;
  if (nodeId) std::copy(m.nodeId.begin(), m.nodeId.end(), nodeId);
  if (conn) std::copy(m.conn.begin(), m.conn.end(), conn);
  if (eIJK) std::copy(m.eIJK.begin(), m.eIJK.end(), eIJK);
  if (colStart) std::copy(m.colStart.begin(), m.colStart.end(), colStart);
  if (cellElems) std::copy(m.cellElems.begin(), m.cellElems.end(), cellElems);
  if (coords) std::copy(m.coords.begin(), m.coords.end(), coords);
  if (constr) std::copy(o->M.constraints.begin(), o->M.constraints.end(), constr);
  if (eGroup) std::copy(m.eGroup.begin(), m.eGroup.end(), eGroup);
}

// Step data per property set: kind (0 homogeneous, 1 layered); D (36) + s0 (6) or W (108) + V (18);
// born: load on/off. Assembles K (full block CSR) and the load; stage sets element birth.
void orc_assemble(orc_model* o, int stage, const int* psetLayered, const double* D, const double* s0,
                  const double* W, const double* V, const int* psetBorn, double* rhs, int noConstraints) {
  Model& M = o->M;
  M.stage = stage;
  for (size_t p = 0; p < M.psets.size(); p++) {
    PropSet& ps = M.psets[p];
    ps.layered = psetLayered[p] != 0;
    if (ps.layered) { std::copy(W + 108 * p, W + 108 * p + 108, ps.W); std::copy(V + 18 * p, V + 18 * p + 18, ps.V); }
    else { std::copy(D + 36 * p, D + 36 * p + 36, ps.D); std::copy(s0 + 6 * p, s0 + 6 * p + 6, ps.s0); }
    ps.born = psetBorn[p] != 0;
  }
  assembleStep(M, rhs, noConstraints != 0);
}

void orc_get_bcsr(orc_model* o, int* rowPtr, int* col, double* val, unsigned char* isC) {
  const Model& M = o->M;
  if (rowPtr) std::copy(M.pattern.rowPtr.begin(), M.pattern.rowPtr.end(), rowPtr);
  if (col) std::copy(M.pattern.col.begin(), M.pattern.col.end(), col);
  if (val) std::copy(M.val.begin(), M.val.end(), val);
  if (isC) { for (int i = 0; i < M.ndof; i++) isC[i] = M.isConstrained.empty() ? 0 : M.isConstrained[i]; }
}

void orc_matvec(orc_model* o, const double* x, double* y) { fullMatVec(o->M.pattern, o->M.val.data(), x, y); }

// precond: 0 MG, 1 IC(0). info (16 doubles): iters, relres, converged, iters0, ms, pcMs, precond, rebuilt,
// warm, fallback, colJitter, shellJitter, levels. key: -1 = none (10-solver.js:937).
int orc_solve(orc_model* o, const double* f, double* u, double tol, int maxit, int precond, long key, double* info) {
  try {
    LinearSolver& S = *o->solver;
    S.tol = tol; S.maxit = maxit;
    if (precond != S.precondKind) { S.precondKind = precond; S.needRebuild = true; }
    SolveInfo in;
    S.solve(f, u, key, in);
    const double vals[16] = {(double)in.iters, in.relres, (double)in.converged, in.iters0, in.ms, in.pcMs, (double)in.precond, (double)in.rebuilt,
                             (double)in.warm, (double)in.fallback, (double)in.colJitter, (double)in.shellJitter, (double)in.levels, 0, 0, 0};
    std::copy(vals, vals + 16, info);
    return 0;
  } catch (std::exception& e) { o->err = e.what(); return 1; }
}

void orc_clear_warm(orc_model* o) { o->solver->basis.clear(); }

// ---- bump submodel -------------------------------------------------------------------------------
struct orc_sub { std::unique_ptr<Submodel> S; std::string err; };

// anand: the 10 Anand constants (A, QR, xi, m, shat, n, h0, a, s0, nu); tables on the 1 degC grid
// (381 points): solder E/F, underfill E/F, silicon F, substrate slice D (36 per point) and F (3
// per point); siD the silicon stiffness (36)
orc_sub* orc_sub_create(int nx, int ny, int nz, const double* xs, const double* ys, const double* zs, const int* cellMat,
                        int nglob, int nt, const double* ts, const double* fields, const double* u25, int nb, const int* bGlob,
                        const double* bW, const double* anand, const double* solderE, const double* solderF, int elasticSolder,
                        const double* ufE, const double* ufF, double ufNu, const double* siD, const double* siF, const double* subD,
                        const double* subF, double nuMax, double zt, double zaf, int uniform, double density, double nuMaxGlobal,
                        int nsec, const double* secZ, const double* secD, const double* secF) {
  SubInput in;
  in.nx = nx; in.ny = ny; in.nz = nz;
  in.xs.assign(xs, xs + nx); in.ys.assign(ys, ys + ny); in.zs.assign(zs, zs + nz);
  in.cellMat.assign(cellMat, cellMat + (size_t)(nx - 1) * (ny - 1) * (nz - 1));
  in.nglob = nglob; in.nt = nt; in.ts.assign(ts, ts + nt);
  in.fields.assign(fields, fields + (size_t)nt * nglob * 3); in.u25.assign(u25, u25 + (size_t)nglob * 3);
  in.bGlob.assign(bGlob, bGlob + 8 * (size_t)nb); in.bW.assign(bW, bW + 8 * (size_t)nb);
  in.anand = AnandParams{anand[0], anand[1], anand[2], anand[3], anand[4], anand[5], anand[6], anand[7], anand[8], anand[9]};
  in.solderE.assign(solderE, solderE + TGRID_N); in.solderF.assign(solderF, solderF + TGRID_N);
  in.elasticSolder = elasticSolder;
  in.ufE.assign(ufE, ufE + TGRID_N); in.ufF.assign(ufF, ufF + TGRID_N); in.ufNu = ufNu;
  in.siD.assign(siD, siD + 36); in.siF.assign(siF, siF + TGRID_N);
  in.subD.assign(subD, subD + 36 * TGRID_N); in.subF.assign(subF, subF + 3 * TGRID_N);
  in.nuMax = nuMax; in.zt = zt; in.zaf = zaf;
  in.uniform = uniform; in.density = density; in.nuMaxGlobal = nuMaxGlobal;
  if (uniform) {
    if (nsec < 1) return nullptr;
    in.nsec = nsec;
    in.secZ.assign(secZ, secZ + 2 * (size_t)nsec);
    in.secD.assign(secD, secD + 36 * (size_t)TGRID_N * nsec);
    in.secF.assign(secF, secF + 3 * (size_t)TGRID_N * nsec);
  }
  auto* o = new orc_sub();
  o->S.reset(new Submodel(in));
  if ((int)o->S->bNodes.size() != nb) { delete o; return nullptr; }
  return o;
}

void orc_sub_destroy(orc_sub* o) { delete o; }
// _elastic of one material over the step from Ta to Tb (subZ: the layer mid-height for the
// substrate slice in the consistency mode): D (36) and the thermal stress increment (6)
void orc_sub_elastic(orc_sub* o, int mat, double subZ, double Ta, double Tb, double* D, double* sth) {
  o->S->elastic(mat, Ta, Tb, D, sth, subZ);
}
// nn, ne, boundary nodes, solder Gauss points
void orc_sub_sizes(orc_sub* o, int* out) {
  int ns = 0;
  for (auto& p : o->S->anand) if (p) ns++;
  out[0] = o->S->m.nn; out[1] = o->S->m.ne; out[2] = (int)o->S->bNodes.size(); out[3] = ns;
}
// one stepTo; returns converged, writes the Newton count and the largest plastic increment
int orc_sub_step(orc_sub* o, double T, double dt, int* newton, double* dMax) { return o->S->stepTo(T, dt, newton, dMax) ? 1 : 0; }
void orc_sub_get_u(orc_sub* o, double* u) { std::copy(o->S->u.begin(), o->S->u.end(), u); }
// W and ebar of every solder Gauss point (element-major)
void orc_sub_get_points(orc_sub* o, double* W, double* ebar) {
  int q = 0;
  for (auto& p : o->S->anand) if (p) { W[q] = p->W; ebar[q] = p->ebar; q++; }
}
int orc_sub_run(orc_sub* o, int nsteps, const double* t, const double* T, const int* cycle, const int* phase, int cycles, double cphi,
                double sphi, double* out, double* perCycle, double* loop, int maxSnaps, int* nSnaps, double* snapMeta, float* snapSig) {
  try {
    o->S->run(nsteps, t, T, cycle, phase, cycles, cphi, sphi, out, perCycle, loop, maxSnaps, nSnaps, snapMeta, snapSig);
    return 0;
  } catch (std::exception& e) { o->err = e.what(); return 1; }
}

// _stressSnapshot of the current state at temperature T (48 floats per element)
void orc_sub_stress_snapshot(orc_sub* o, double T, float* out) { o->S->stressSnapshot(T, out); }

// pc.apply(r, z) of the preconditioner the last solve built (scaled space); 1 when none
int orc_pc_apply(orc_model* o, const double* r, double* z) {
  if (!o->solver->pc) return 1;
  o->solver->pc->apply(r, z);
  return 0;
}

// MG level sizes after a solve: per level (nx, ny, nn, b)
int orc_mg_levels(orc_model* o, int* out, int cap) {
  auto* mg = dynamic_cast<MultigridPC*>(o->solver->pc.get());
  if (!mg) return 0;
  int L = (int)mg->levels.size();
  for (int l = 0; l < L && l < cap; l++) { out[4 * l] = mg->levels[l]->nx; out[4 * l + 1] = mg->levels[l]->ny; out[4 * l + 2] = mg->levels[l]->nn; out[4 * l + 3] = mg->levels[l]->b; }
  return L;
}

// aggregate index per fine node (level 0 -> shell level 1) of the last preconditioner
int orc_mg_node_agg(orc_model* o, int* out) {
  auto* mg = dynamic_cast<MultigridPC*>(o->solver->pc.get());
  if (!mg) return 0;
  std::copy(mg->levels[0]->nodeAgg.begin(), mg->levels[0]->nodeAgg.end(), out);
  return (int)mg->levels[0]->nodeAgg.size();
}

// ---- element-level entry points --------------------------------------------------------
void orc_shape_matrices(const double* Wst, const double* D, double* M) { shapeMatrices(Wst, D, M); }
void orc_element_k33(double hx, double hy, double hz, const double* M, double* K) { elementK33Fast(hx, hy, hz, M, K); }
void orc_element_fth(double hx, double hy, double hz, const double* Sst, const double* s0, double* f) { elementFth(hx, hy, hz, Sst, s0, f); }
void orc_condense33(const double* K, const double* f, double* Kc, double* fc, double* X) { condense33(K, f, Kc, fc, X); }
void orc_general_element(const double* X, const double* D, double* Kc, double* Xc) { generalElement(X, D, Kc, Xc); }
void orc_box_derivs(double hx, double hy, double hz, double xi, double eta, double zeta, double* dx, double* dy, double* dz) { boxDerivs(hx, hy, hz, xi, eta, zeta, dx, dy, dz); }
void orc_general_derivs(const double* X, double xi, double eta, double zeta, double* dx, double* dy, double* dz) {
  double J[9] = {0}, J0i[9];
  for (int a = 0; a < 8; a++) for (int j = 0; j < 3; j++) {
    J[j] += HEX_XI[a] * 0.125 * X[3 * a + j]; J[3 + j] += HEX_ETA[a] * 0.125 * X[3 * a + j]; J[6 + j] += HEX_ZETA[a] * 0.125 * X[3 * a + j];
  }
  const double det0 = inv3(J, J0i);
  generalDerivs(X, xi, eta, zeta, J0i, det0, dx, dy, dz);
}
int orc_chol_dense(double* A, int n, double rel) { return cholDense(A, n, rel); }

// ---- Anand entry points ------------------------------------------------------------------
// params: A, QR, xi, m, shat, n, h0, a, s0, nu; Etab: E(T) on the 1 degC grid (-80..300, MPa)
// state (12): ep[6], s, ebar, W, sigEq, lastD, (unused); updated only when commit != 0
double orc_anand_step(const double* params, const double* Etab, double* state, const double* eps, double T, double dt,
                      double* sig, double* D, int wantTangent, int commit) {
  AnandParams P{params[0], params[1], params[2], params[3], params[4], params[5], params[6], params[7], params[8], params[9]};
  AnandPoint pt(P, Etab);
  for (int i = 0; i < 6; i++) pt.ep[i] = state[i];
  pt.s = state[6]; pt.ebar = state[7]; pt.W = state[8]; pt.sigEq = state[9]; pt.lastD = state[10];
  double Dl[36];
  const double d = pt.step(eps, T, dt, sig, D ? D : Dl, wantTangent != 0, nullptr);
  if (commit) pt.commit();
  for (int i = 0; i < 6; i++) state[i] = pt.ep[i];
  state[6] = pt.s; state[7] = pt.ebar; state[8] = pt.W; state[9] = pt.sigEq; state[10] = pt.lastD;
  return d;
}

// stepSeriesColumn (13-fatigue.js:178-206) of one point: the cap's strain eps (guess in, solution
// out) for the prescribed column-average (zz, yz, zx) strains tz, cap fraction fs and pillar
// compliances Cp; the state as in orc_anand_step; returns the plastic increment
double orc_anand_series_step(const double* params, const double* Etab, double* state, double* eps, const double* tz, double fs,
                             const double* Cp, double T, double dt, double* sig, double* D, int commit) {
  AnandParams P{params[0], params[1], params[2], params[3], params[4], params[5], params[6], params[7], params[8], params[9]};
  AnandPoint pt(P, Etab);
  for (int i = 0; i < 6; i++) pt.ep[i] = state[i];
  pt.s = state[6]; pt.ebar = state[7]; pt.W = state[8]; pt.sigEq = state[9]; pt.lastD = state[10];
  const double d = pt.stepSeriesColumn(eps, tz, fs, Cp, T, dt, sig, D, nullptr);
  if (commit) pt.commit();
  for (int i = 0; i < 6; i++) state[i] = pt.ep[i];
  state[6] = pt.s; state[7] = pt.ebar; state[8] = pt.W; state[9] = pt.sigEq; state[10] = pt.lastD;
  return d;
}

// anandUniaxial (13-fatigue.js:252-272): returns the final stress
double orc_anand_uniaxial(const double* params, const double* Etab, double T, double rate, double epsMax, int nsteps) {
  AnandParams P{params[0], params[1], params[2], params[3], params[4], params[5], params[6], params[7], params[8], params[9]};
  AnandPoint pt(P, Etab);
  double eps[6] = {0}, sig[6], D[36];
  const double dt = epsMax / rate / nsteps;
  double lat = 0, last = 0;
  for (int k = 1; k <= nsteps; k++) {
    eps[0] = rate * dt * k;
    for (int it = 0; it < 30; it++) {
      eps[1] = eps[2] = lat;
      pt.step(eps, T, dt, sig, D, true, nullptr);
      const double r = sig[1];
      if (std::fabs(r) < 1e-9 * std::max(1.0, std::fabs(sig[0]))) break;
      const double dr = D[7] + D[8];
      lat -= r / dr;
    }
    pt.commit();
    last = sig[0];
  }
  return last;
}

// The per-site loop of screenJoints (13-fatigue.js:395-451): table (nsites x ntemps x 6) of
// bump-layer total strains at the cycling temperatures `temps`, the time history (t, T, cycle,
// phase) of cycleHistory, thermal strain table Ftab on the 1 degC grid. Without a pillar
// (pEtab == nullptr) every joint is a free-standing solder column (stepColumn); with one it is a
// solder cap of height fraction fs on an elastic pillar (E table pEtab, Poisson ratio pNu,
// thermal strain table pFtab) in series (stepSeriesColumn, screenDdi :369-376). Outputs dW,
// dE, stab per site (NaN where the table is not finite).
static void screenLoop(const double* params, const double* Etab, const double* Ftab,
                       int nsites, int ntemps, const double* temps, const double* table,
                       int nsteps, const double* th, const double* Th, const int* cycle, const int* phase, int cycles,
                       double fs, double pNu, const double* pEtab, const double* pFtab,
                       double* dW, double* dE, double* stab) {
  AnandParams P{params[0], params[1], params[2], params[3], params[4], params[5], params[6], params[7], params[8], params[9]};
  AnandPoint pt(P, Etab);
  const double nu = P.nu;
  const int IP[3] = {0, 1, 3};
  const bool pillar = pEtab != nullptr;
  if (!pillar) fs = 1;
  int i25 = -1;
  for (int i = 0; i < ntemps; i++) if (temps[i] == 25) { i25 = i; break; }
  std::vector<int> wi(nsteps); dvec wt(nsteps), Fth(nsteps), Cps(pillar ? 3 * nsteps : 0), Fp(pillar ? nsteps : 0);
  std::vector<StepK> kc(nsteps);
  for (int k = 0; k < nsteps; k++) {
    // findInterval (01-util.js:12-22)
    int i;
    if (Th[k] <= temps[0]) i = 0;
    else if (Th[k] >= temps[ntemps - 1]) i = ntemps - 2;
    else { int lo = 0, hi = ntemps - 1; while (hi - lo > 1) { const int mid = (lo + hi) >> 1; if (temps[mid] <= Th[k]) lo = mid; else hi = mid; } i = lo; }
    wi[k] = i;
    const double t = (Th[k] - temps[i]) / (temps[i + 1] - temps[i]);
    wt[k] = t < 0 ? 0 : (t > 1 ? 1 : t);
    Fth[k] = gridAt(Ftab, Th[k]) - gridAt(Ftab, 25);
    if (k > 0) kc[k] = pt.stepConstants(Th[k], th[k] - th[k - 1]);
    if (pillar) {   // :410-414
      const double Ep = gridAt(pEtab, Th[k]), Gp = Ep / (2 * (1 + pNu));
      Cps[3 * k] = 1 / Ep; Cps[3 * k + 1] = Cps[3 * k + 2] = 1 / Gp;
      Fp[k] = gridAt(pFtab, Th[k]) - gridAt(pFtab, 25);
    }
  }
  dvec Wc(cycles + 1), Ec(cycles + 1);
  double eps[6], e25[6], e1[3], e2[3], s1[6], s2[6], tz[3], sig[6], D[36];
  for (int q = 0; q < nsites; q++) {
    const size_t base = (size_t)q * ntemps * 6;
    dW[q] = dE[q] = stab[q] = NAN;
    if (!std::isfinite(table[base])) continue;
    pt.reset();
    for (int c = 0; c < 6; c++) e25[c] = i25 >= 0 ? table[base + i25 * 6 + c] : 0;
    std::fill(Wc.begin(), Wc.end(), 0.0); std::fill(Ec.begin(), Ec.end(), 0.0);
    for (auto& v : eps) v = 0;
    for (int c = 0; c < 3; c++) { e1[c] = 0; e2[c] = 0; }
    for (int c = 0; c < 6; c++) { s1[c] = 0; s2[c] = 0; }
    for (int k = 1; k < nsteps; k++) {
      const size_t a = base + (size_t)wi[k] * 6, b = a + 6; const double t = wt[k];
      auto lay = [&](int c) { return table[a + c] + t * (table[b + c] - table[a + c]) - e25[c]; };
      if (pillar) {
        tz[0] = lay(2) - fs * Fth[k] - (1 - fs) * Fp[k]; tz[1] = lay(4); tz[2] = lay(5);
        if (k > 2 && phase[k] == phase[k - 1]) for (int c = 0; c < 6; c++) eps[c] = 2 * s1[c] - s2[c];
        pt.stepSeriesColumn(eps, tz, fs, Cps.data() + 3 * k, Th[k], kc[k].dt, sig, D, &kc[k]);
        for (int c = 0; c < 6; c++) { s2[c] = s1[c]; s1[c] = eps[c]; }
      } else {
        const double ez = lay(2) - Fth[k];
        if (k > 2 && phase[k] == phase[k - 1]) for (int r = 0; r < 3; r++) eps[IP[r]] = 2 * e1[r] - e2[r];
        else { eps[0] -= nu * (ez - eps[2]); eps[1] -= nu * (ez - eps[2]); }
        eps[2] = ez; eps[4] = lay(4); eps[5] = lay(5);
        pt.stepColumn(eps, Th[k], kc[k].dt, sig, D, &kc[k]);
      }
      pt.commit();
      for (int r = 0; r < 3; r++) { e2[r] = e1[r]; e1[r] = eps[IP[r]]; }
      const int cyc = cycle[k];
      Wc[cyc] = pt.W; Ec[cyc] = pt.ebar;
    }
    const int nc = cycles;
    dW[q] = Wc[nc] - Wc[nc - 1];
    dE[q] = Ec[nc] - Ec[nc - 1];
    stab[q] = nc >= 2 ? std::fabs((Wc[nc] - Wc[nc - 1]) - (Wc[nc - 1] - Wc[nc - 2])) / std::max(Wc[nc] - Wc[nc - 1], 1e-30) : NAN;
  }
}

void orc_anand_screen(const double* params, const double* Etab, const double* Ftab,
                      int nsites, int ntemps, const double* temps, const double* table,
                      int nsteps, const double* th, const double* Th, const int* cycle, const int* phase, int cycles,
                      double* dW, double* dE, double* stab) {
  screenLoop(params, Etab, Ftab, nsites, ntemps, temps, table, nsteps, th, Th, cycle, phase, cycles, 1, 0, nullptr, nullptr, dW, dE, stab);
}

// screenDdi's joints: a solder cap of height fraction fs on an elastic pillar (pillar Poisson
// ratio pNu, E and thermal strain tables pEtab, pFtab on the 1 degC grid)
void orc_anand_screen_pillar(const double* params, const double* Etab, const double* Ftab,
                             int nsites, int ntemps, const double* temps, const double* table,
                             int nsteps, const double* th, const double* Th, const int* cycle, const int* phase, int cycles,
                             double fs, double pNu, const double* pEtab, const double* pFtab,
                             double* dW, double* dE, double* stab) {
  screenLoop(params, Etab, Ftab, nsites, ntemps, temps, table, nsteps, th, Th, cycle, phase, cycles, fs, pNu, pEtab, pFtab, dW, dE, stab);
}

// ---- element DOF histories and post-processing readers ----------------------------------------
// Model.accumulateStep (qOnly) over nel elements for the last assembled step
void orc_accumulate_q(orc_model* o, const double* du, int nel, const int* elems, double* q) {
  for (int t = 0; t < nel; t++) accumulateQ(o->M, du, elems[t], q + 33 * (size_t)t);
}

// sub-layers of the layered property sets for the stress histories: nsub per property set (0 for
// homogeneous ones), then per sub-layer in set order its z range (2), mean stiffness (36) and
// thermal stress increment (6) of the step assembled last
void orc_set_sublayers(orc_model* o, const int* nsub, const double* subZ, const double* subD, const double* subS0) {
  size_t q = 0;
  for (auto& ps : o->M.psets) {
    const int n = nsub[&ps - &o->M.psets[0]];
    ps.nsub = n;
    ps.subZ.assign(subZ + 2 * q, subZ + 2 * (q + n));
    ps.subD.assign(subD + 36 * q, subD + 36 * (q + n));
    ps.subS0.assign(subS0 + 6 * q, subS0 + 6 * (q + n));
    q += n;
  }
}

// element histories with stresses: state (stride doubles per element) += the step's increment
void orc_accumulate_state(orc_model* o, const double* du, int nel, const int* elems, int stride, double* state) {
  for (int t = 0; t < nel; t++) accumulateState(o->M, du, elems[t], state + (size_t)stride * t);
}

// stress and strain at natural points from the element states (stride doubles per point)
void orc_state_stress(orc_model* o, int np, const int* elem, const double* state, int stride, const double* nat, double* eps,
                      double* sig) {
  for (int t = 0; t < np; t++)
    stateStress(o->M, elem[t], state + (size_t)stride * t, nat + 3 * (size_t)t, eps + 6 * (size_t)t, sig + 6 * (size_t)t);
}

void orc_element_strains(orc_model* o, int np, const int* elem, const double* q, const double* nat, double* eps) {
  for (int t = 0; t < np; t++) elementStrain(o->M, elem[t], q + 33 * (size_t)t, nat + 3 * (size_t)t, eps + 6 * (size_t)t);
}
void orc_fit_plane(int n, const double* x, const double* y, const double* w, double* c3) { fitPlane(n, x, y, w, c3); }
double orc_sample_plane(orc_model* o, const double* u, int k, int comp, double x, double y) { return samplePlane(o->M.mesh, u, k, comp, x, y); }
// out (9): signed, magnitude, sign, sign confidence, plane c0 c1 c2, rmin, rmax
void orc_warpage_jeita(orc_model* o, const double* u, int nb, const double* bx, const double* by, const double* zone, double* out) {
  warpageJEITA(o->M.mesh, u, nb, bx, by, zone, out);
}

const char* orc_last_error(orc_model* o) { return o->err.c_str(); }

}  // extern "C"
