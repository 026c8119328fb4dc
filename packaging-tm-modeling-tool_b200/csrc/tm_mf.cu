// Matrix-free level-0 operator: the stiffness apply y = K x (fullMatVec, src/core/09-assembly.js:151-165)
// and the z-column Gauss-Seidel sweep of the multigrid's solid level (columnSweep solid branch,
// src/core/10-solver.js:512-534, with solveColumn :71-104) computed from the condensed element
// matrices instead of the assembled operator.
//
// The operator that assembleStep scatters (09-assembly.js:392-424) is the sum over the elements e of
// scale_e * Kc(class_e), with scale_e = eScale[e] * (1 or 1e-6 before the element's stage) and Kc
// the condensed 24x24 matrix of the element's class (property set, hx, hy, hz; condense33,
// 07-element.js:88-121). A mesh cell holds at most two superposed elements (cellElems), so every
// cell is given one cell class: the pair (class, scale) of its elements, whose combined matrix
// sum_q scale_q Kc(class_q) is formed on the device once per step. The benchmark package has 46
// element classes and about as many cell classes for 819,200 cells, so the whole table (576
// values per class) stays in L1/L2 and a cell costs 2 bytes of HBM instead of the 243 stored
// values per node of the assembled stencil.
//
// The solver works on the Jacobi-scaled operator with the constraints applied (_scale,
// 10-solver.js:852-866; applyConstraints, 09-assembly.js:445-464): Ks = S K S with the rows and
// columns of constrained DOFs zeroed and their diagonal kept. The kernels read three per-DOF
// vectors: gs (S, zero at constrained DOFs) scales x where it is gathered, os (S) scales the row
// sums, and cd (the kept diagonal) gives the rows of constrained DOFs, y_c = cd_c x_c. Before the
// first solve of a step (the unscaled operator) gs = 1 and os = 1.
//
// Summation order: a node's row is the sum over its (up to 8) cells of the cell matrix rows times
// the cell's 24 gathered values, not the assembled entries' sums, so results agree with the
// assembled apply to rounding (about 1e-16 relative per entry), not bitwise.
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cstring>
#include <map>
#include <tuple>

#include "tm_internal.h"

namespace tmg {

namespace {

constexpr uint16_t MF_NONE = 0xFFFF;
constexpr int MF_MAX_CC = 4096;    // beyond this many cell classes the assembled stencil is used

inline int grid_for(size_t n, int block) { return (int)((n + block - 1) / block); }

// local node order loc of the mesher (06-mesher.js:49): index L <-> offsets (a, b, c) in x, y, z
__host__ __device__ constexpr int loc_a(int L) { return ((L & 3) == 1 || (L & 3) == 2) ? 1 : 0; }
__host__ __device__ constexpr int loc_b(int L) { return (L & 3) >= 2 ? 1 : 0; }
__host__ __device__ constexpr int loc_c(int L) { return L >> 2; }
__host__ __device__ constexpr int loc_of(int a, int b, int c) { return c * 4 + (b ? (a ? 2 : 3) : (a ? 1 : 0)); }

// ---- per step: combined cell matrices --------------------------------------------------------------
// ccK[cc] = s0 Kc(c0) + s1 Kc(c1) (the second term only for superposed cells), FP64 and FP32
__global__ void k_cc_combine(int ncc, const int* __restrict__ info, const double* __restrict__ scale, const double* __restrict__ clsKc,
                             double* __restrict__ ccK, float* __restrict__ ccK32) {
  const int cc = blockIdx.x;
  if (cc >= ncc) return;
  const int c0 = info[2 * cc], c1 = info[2 * cc + 1];
  const double s0 = scale[2 * cc], s1 = scale[2 * cc + 1];
  for (int r = threadIdx.x; r < 576; r += blockDim.x) {
    double v = s0 * clsKc[(size_t)c0 * 576 + r];
    if (c1 >= 0) v += s1 * clsKc[(size_t)c1 * 576 + r];
    ccK[(size_t)cc * 576 + r] = v;
    ccK32[(size_t)cc * 576 + r] = (float)v;
  }
}

// per DOF: gs (gather scale), os (row scale), cd (kept diagonal of constrained rows, read from the
// assembled operator's diagonal block at slot-major position pos), FP64 and FP32
__global__ void k_mf_scales(int nn, int S, const int* __restrict__ pos, const uint8_t* __restrict__ isC, const double* __restrict__ s,
                            const double* __restrict__ val, double* __restrict__ gs, double* __restrict__ os, double* __restrict__ cd,
                            float* __restrict__ gs32, float* __restrict__ os32, float* __restrict__ cd32) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= 3 * nn) return;
  const int n = t / 3, p = t % 3;
  const double sv = s ? s[t] : 1.0;
  const bool con = isC[t] != 0;
  const double g = con ? 0.0 : sv;
  const double d = con ? val[((size_t)SLOT_SELF * 9 + 4 * p) * S + pos[n]] : 0.0;
  gs[t] = g; os[t] = sv; cd[t] = d;
  gs32[t] = (float)g; os32[t] = (float)sv; cd32[t] = (float)d;
}

// ---- the row of one node from its 8 cells ---------------------------------------------------------
template <class T>
struct KRow;
template <>
struct KRow<float> {
  // the 24 values of one row of a cell matrix
  static __device__ __forceinline__ void load(const float* __restrict__ K, float (&k)[24]) {
    const float4* q = reinterpret_cast<const float4*>(K);
#pragma unroll
    for (int i = 0; i < 6; i++) {
      const float4 v = __ldg(q + i);
      k[4 * i] = v.x; k[4 * i + 1] = v.y; k[4 * i + 2] = v.z; k[4 * i + 3] = v.w;
    }
  }
};
template <>
struct KRow<double> {
  static __device__ __forceinline__ void load(const double* __restrict__ K, double (&k)[24]) {
    const double2* q = reinterpret_cast<const double2*>(K);
#pragma unroll
    for (int i = 0; i < 12; i++) {
      const double2 v = __ldg(q + i);
      k[2 * i] = v.x; k[2 * i + 1] = v.y;
    }
  }
};

// acc += the node's rows of K x. Staged gs*x is stored by component (structure of arrays):
// component q of the node at staged (kk, ii, jj) is xs[q*NS + (kk*PI + ii)*PJ + jj], so a warp whose
// lanes take consecutive (or every other) jj reads 32 different banks. (ii, jj, kk): the node's
// staged coordinates; (ci0, cj0, ck0): the staged coordinates of cell (i-1, j-1, k-1), cells stored at
// (ck*CI + ci)*CJ + cj. Per cell layer c the node's 18 neighbours on its two node planes are loaded
// once into registers and serve that layer's four cells (the cell whose corner (1-a, 1-b, 1-c) is the
// node, its 8 nodes in the local order of the element matrix).
template <class T, int PI, int PJ, int CI, int CJ>
__device__ __forceinline__ void node_row(const T* __restrict__ xs, int NS, const uint16_t* __restrict__ cls, const T* __restrict__ ccK,
                                         int ii, int jj, int kk, int ci0, int cj0, int ck0, T (&acc)[3]) {
#pragma unroll
  for (int c = 0; c < 2; c++) {
    T xv[2][3][3][3];
#pragma unroll
    for (int dk = 0; dk < 2; dk++)
#pragma unroll
      for (int di = 0; di < 3; di++)
#pragma unroll
        for (int dj = 0; dj < 3; dj++) {
          const int at = ((kk - 1 + c + dk) * PI + ii - 1 + di) * PJ + jj - 1 + dj;
#pragma unroll
          for (int q = 0; q < 3; q++) xv[dk][di][dj][q] = xs[q * NS + at];
        }
#pragma unroll
    for (int b = 0; b < 2; b++)
#pragma unroll
      for (int a = 0; a < 2; a++) {
        const int cc = cls[((ck0 + c) * CI + ci0 + a) * CJ + cj0 + b];
        if (cc == MF_NONE) continue;
        const int Lrow = loc_of(1 - a, 1 - b, 1 - c);
        const T* K = ccK + (size_t)cc * 576 + 3 * Lrow * 24;
#pragma unroll
        for (int p = 0; p < 3; p++) {
          T k[24];
          KRow<T>::load(K + 24 * p, k);
          T s = 0;
#pragma unroll
          for (int M = 0; M < 8; M++)
#pragma unroll
            for (int q = 0; q < 3; q++) s += k[3 * M + q] * xv[loc_c(M)][a + loc_a(M)][b + loc_b(M)][q];
          acc[p] += s;
        }
      }
  }
}

// ---- staging of a box of nodes and cells into shared memory -----------------------------------------
// Items are walked with the node planes fastest (consecutive node ids of a column, coalesced). Each
// thread keeps SB items in flight: first all their node ids, then all their x and gs, so a thread
// waits for two rounds of loads per SB items instead of two per item.
constexpr int SB = 8;

// gs*x of the box of PI x PJ node columns from (i0, j0), planes k0 .. k0+np-1, by component into
// xs[q*NS + (kk*PI + ii)*PJ + jj], NS = np*PI*PJ (zero outside the mesh and where no node exists);
// when ids is not null, the node ids (-1 for none) into ids[(kk*PI + ii)*PJ + jj]
template <class T, int PI, int PJ>
__device__ __forceinline__ void stage_nodes(int nx, int ny, int nz, int i0, int j0, int k0, int np, const int* __restrict__ nodeId,
                                            const T* __restrict__ x, const T* __restrict__ gs, T* xs, int* ids) {
  const int total = PI * PJ * np;
  for (int t0 = threadIdx.x; t0 < total; t0 += SB * blockDim.x) {
    int n[SB];
#pragma unroll
    for (int u = 0; u < SB; u++) {
      const int t = t0 + u * blockDim.x;
      n[u] = -1;
      if (t < total) {
        const int kk = t % np, col = t / np, jj = col % PJ, ii = col / PJ;
        const int i = i0 + ii, j = j0 + jj, k = k0 + kk;
        if (i >= 0 && i < nx && j >= 0 && j < ny && k >= 0 && k < nz) n[u] = nodeId[((size_t)i * ny + j) * nz + k];
      }
    }
    T v[SB][3];
#pragma unroll
    for (int u = 0; u < SB; u++) {
      const size_t o = 3 * (size_t)(n[u] < 0 ? 0 : n[u]);
#pragma unroll
      for (int q = 0; q < 3; q++) v[u][q] = n[u] >= 0 ? x[o + q] * gs[o + q] : (T)0;
    }
#pragma unroll
    for (int u = 0; u < SB; u++) {
      const int t = t0 + u * blockDim.x;
      if (t >= total) break;
      const int kk = t % np, col = t / np, jj = col % PJ, ii = col / PJ;
      const int at = (kk * PI + ii) * PJ + jj;
      xs[at] = v[u][0]; xs[total + at] = v[u][1]; xs[2 * total + at] = v[u][2];
      if (ids) ids[at] = n[u];
    }
  }
}

// cell classes of the box of CI x CJ cell columns from (i0, j0), layers k0 .. k0+nl-1, into
// cls[(kk*CI + ci)*CJ + cj] (MF_NONE outside the mesh)
template <int CI, int CJ>
__device__ __forceinline__ void stage_cells(int nx, int ny, int nz, int i0, int j0, int k0, int nl, const uint16_t* __restrict__ cellCls,
                                            uint16_t* cls) {
  const int ncy = ny - 1, ncz = nz - 1;
  const int total = CI * CJ * nl;
  for (int t0 = threadIdx.x; t0 < total; t0 += SB * blockDim.x) {
    uint16_t v[SB];
#pragma unroll
    for (int u = 0; u < SB; u++) {
      const int t = t0 + u * blockDim.x;
      v[u] = MF_NONE;
      if (t < total) {
        const int kk = t % nl, col = t / nl, cj = col % CJ, ci = col / CJ;
        const int i = i0 + ci, j = j0 + cj, k = k0 + kk;
        if (i >= 0 && i < nx - 1 && j >= 0 && j < ncy && k >= 0 && k < ncz) v[u] = cellCls[((size_t)i * ncy + j) * ncz + k];
      }
    }
#pragma unroll
    for (int u = 0; u < SB; u++) {
      const int t = t0 + u * blockDim.x;
      if (t >= total) break;
      const int kk = t % nl, col = t / nl, cj = col % CJ, ci = col / CJ;
      cls[(kk * CI + ci) * CJ + cj] = v[u];
    }
  }
}

// ---- apply over all nodes: tiles of MF_TI x MF_TJ node columns and a slab of ks node planes --------
// A warp takes one row of the tile's 32 node columns in one plane (lane = jj): its lanes read
// consecutive words of the staged x and the same cell layer, so the class-table loads are uniform.
constexpr int MF_TI = 4, MF_TJ = 32;
constexpr int MF_PI = MF_TI + 2, MF_PJ = MF_TJ + 2;       // staged node columns (one halo column each side)
constexpr int MF_CI = MF_TI + 1, MF_CJ = MF_TJ + 1;       // staged cell columns
constexpr int MF_THREADS = 256;
constexpr int MF_PLANES = MF_THREADS / 32 / MF_TI;        // planes per pass of the CTA's warps

template <class T>
inline size_t mf_apply_smem(int ks) {
  const size_t nodes = (size_t)(ks + 2) * MF_PI * MF_PJ;
  return nodes * 3 * sizeof(T) + nodes * sizeof(int) + (size_t)(ks + 1) * MF_CI * MF_CJ * sizeof(uint16_t) + 16;
}

struct MfDims {
  int nx, ny, nz;      // node grid lines
  int tilesI, tilesJ, slabs, ks;
};

template <class T, bool RES>
__global__ void __launch_bounds__(MF_THREADS) k_mf_apply(MfDims d, const int* __restrict__ nodeId, const uint16_t* __restrict__ cellCls,
                                                         const T* __restrict__ ccK, const T* __restrict__ gs, const T* __restrict__ os,
                                                         const T* __restrict__ cd, const T* __restrict__ x, const T* __restrict__ b,
                                                         T* __restrict__ y) {
  extern __shared__ __align__(16) unsigned char smraw[];
  const int ks = d.ks;
  const int np = ks + 2;
  const int NS = np * MF_PI * MF_PJ;
  T* xs = reinterpret_cast<T*>(smraw);
  int* ids = reinterpret_cast<int*>(xs + 3 * (size_t)NS);
  uint16_t* cls = reinterpret_cast<uint16_t*>(ids + NS);
  int blk = blockIdx.x;
  const int slab = blk % d.slabs; blk /= d.slabs;
  const int tj = blk % d.tilesJ, ti = blk / d.tilesJ;
  const int i0 = ti * MF_TI, j0 = tj * MF_TJ, k0 = slab * ks;
  // gs*x and the node ids of the tile's node columns plus one halo column and plane on every side,
  // and the cell classes of cells (i0-1 .. i0+TI-1) x (j0-1 ..) x (k0-1 .. k0+ks-1)
  stage_nodes<T, MF_PI, MF_PJ>(d.nx, d.ny, d.nz, i0 - 1, j0 - 1, k0 - 1, np, nodeId, x, gs, xs, ids);
  stage_cells<MF_CI, MF_CJ>(d.nx, d.ny, d.nz, i0 - 1, j0 - 1, k0 - 1, ks + 1, cellCls, cls);
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int ii = warp % MF_TI, jj = lane;
  const int i = i0 + ii, j = j0 + jj;
  if (i >= d.nx || j >= d.ny) return;
  for (int kk = warp / MF_TI; kk < ks; kk += MF_PLANES) {
    const int k = k0 + kk;
    if (k >= d.nz) break;
    const int n = ids[((kk + 1) * MF_PI + ii + 1) * MF_PJ + jj + 1];
    if (n < 0) continue;
    T acc[3] = {0, 0, 0};
    // staged node coordinates of the node: (ii+1, jj+1, kk+1); of cell (i-1, j-1, k-1): (ii, jj, kk)
    node_row<T, MF_PI, MF_PJ, MF_CI, MF_CJ>(xs, NS, cls, ccK, ii + 1, jj + 1, kk + 1, ii, jj, kk, acc);
    const size_t o = 3 * (size_t)n;
#pragma unroll
    for (int p = 0; p < 3; p++) {
      const T g = gs[o + p];
      const T v = g != (T)0 ? os[o + p] * acc[p] : cd[o + p] * x[o + p];
      y[o + p] = RES ? b[o + p] - v : v;
    }
  }
}

// ---- one colour of the level-0 sweep: residual rows, then the column solves -----------------------------
// Residual: a CTA takes one colour row of RS_SC colour columns (i = pi + 2 tr, j = pj + 2 (RS_SC tc + c))
// over all planes; their neighbours span 3 x (2 RS_SC + 1) node columns. Lanes 0-15 take the 16
// columns at one plane (every other staged column: 16 banks), lanes 16-31 the next plane (an odd
// plane stride away: the other 16 banks). r = b - Ks x goes to a global buffer in node order.
constexpr int RS_SC = 16;
constexpr int RS_PI = 3, RS_PJ = 2 * RS_SC + 1, RS_CI = 2, RS_CJ = 2 * RS_SC;
constexpr int RS_THREADS = 256;

template <class T>
inline size_t mf_resid_smem(int nz) {
  const size_t nodes = (size_t)(nz + 2) * RS_PI * RS_PJ;
  return nodes * 3 * sizeof(T) + (size_t)(nz + 1) * RS_CI * RS_CJ * sizeof(uint16_t) + (size_t)RS_SC * nz * sizeof(int) + 32;
}

struct MfColDims {
  int nx, ny, nz;
  int pi, pj;          // colour parities
  int rows, cols;      // colour rows / columns of the colour
  int tilesJ;          // tiles along the colour columns
};

template <class T>
__global__ void __launch_bounds__(RS_THREADS) k_mf_resid(MfColDims d, const int* __restrict__ nodeId, const uint16_t* __restrict__ cellCls,
                                                         const T* __restrict__ ccK, const T* __restrict__ gs, const T* __restrict__ os,
                                                         const T* __restrict__ cd, const T* __restrict__ b, const T* __restrict__ x,
                                                         T* __restrict__ r) {
  extern __shared__ __align__(16) unsigned char smraw[];
  const int nz = d.nz;
  const int NS = (nz + 2) * RS_PI * RS_PJ;
  T* xs = reinterpret_cast<T*>(smraw);
  uint16_t* cls = reinterpret_cast<uint16_t*>(xs + 3 * (size_t)NS);
  int* nid = reinterpret_cast<int*>(smraw + ((3 * (size_t)NS * sizeof(T) + (size_t)(nz + 1) * RS_CI * RS_CJ * sizeof(uint16_t) + 15) / 16) * 16);
  const int tr = blockIdx.x / d.tilesJ, tc = blockIdx.x % d.tilesJ;
  const int i = d.pi + 2 * tr;
  const int iLo = i - 1, jLo = d.pj + 2 * RS_SC * tc - 1;   // first staged node column
  // the node ids of the tile's columns (-1: none), SB per thread in flight
  for (int t0 = threadIdx.x; t0 < RS_SC * nz; t0 += SB * blockDim.x) {
    int n[SB];
#pragma unroll
    for (int u = 0; u < SB; u++) {
      const int t = t0 + u * blockDim.x;
      n[u] = -1;
      if (t < RS_SC * nz) {
        const int c = t / nz, k = t % nz;
        if (RS_SC * tc + c < d.cols) n[u] = nodeId[((size_t)i * d.ny + jLo + 1 + 2 * c) * nz + k];
      }
    }
#pragma unroll
    for (int u = 0; u < SB; u++) {
      const int t = t0 + u * blockDim.x;
      if (t < RS_SC * nz) nid[t] = n[u];
    }
  }
  // node plane k is staged at k+1, cell layer k at k+1
  stage_nodes<T, RS_PI, RS_PJ>(d.nx, d.ny, nz, iLo, jLo, -1, nz + 2, nodeId, x, gs, xs, nullptr);
  stage_cells<RS_CI, RS_CJ>(d.nx, d.ny, nz, iLo, jLo, -1, nz + 1, cellCls, cls);
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int c = lane & (RS_SC - 1), jj = 1 + 2 * c;
  for (int k = 2 * warp + (lane >> 4); k < nz; k += 2 * (RS_THREADS / 32)) {
    const int n = nid[c * nz + k];
    if (n < 0) continue;
    T acc[3] = {0, 0, 0};
    // node (i, j, k) at staged (1, jj, k+1); cell (i-1, j-1, k-1) at staged (0, jj-1, k)
    node_row<T, RS_PI, RS_PJ, RS_CI, RS_CJ>(xs, NS, cls, ccK, 1, jj, k + 1, 0, jj - 1, k, acc);
    const size_t o = 3 * (size_t)n;
#pragma unroll
    for (int p = 0; p < 3; p++) {
      const T g = gs[o + p];
      r[o + p] = b[o + p] - (g != (T)0 ? os[o + p] * acc[p] : cd[o + p] * x[o + p]);
    }
  }
}

// Column solves: a warp per column of the colour's list; lane l holds the positions l, l+32, ... of
// the column (its factors, 15 of the 18 values, and its residual rows, coalesced loads), and the
// block-tridiagonal forward and backward substitutions of solveColumn (10-solver.js:71-104) run down
// and up the column with the neighbour's values broadcast by warp shuffles. x += dx (x = dx on the
// cycle's first sweep, whose residual is b itself).
constexpr int CS_MAXS = 4;   // up to 128 nodes per column
template <class T>
__global__ void __launch_bounds__(256) k_col_solve(int ncols, const int* __restrict__ colPos, const int* __restrict__ posNode,
                                                   const T* __restrict__ F, const T* __restrict__ r, T* __restrict__ x, int zeroGuess) {
  const int lane = threadIdx.x & 31;
  const int q = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (q >= ncols) return;
  const int p0 = colPos[q], len = colPos[q + 1] - p0;
  T f[CS_MAXS][15], v[CS_MAXS][3];
  int nd[CS_MAXS];
#pragma unroll
  for (int s = 0; s < CS_MAXS; s++) {
    const int pos = 32 * s + lane;
    nd[s] = -1;
    if (pos < len) {
      const T* fp = F + 18 * (size_t)(p0 + pos);
      f[s][0] = fp[1]; f[s][1] = fp[2]; f[s][2] = fp[3]; f[s][3] = fp[5]; f[s][4] = fp[6]; f[s][5] = fp[7];
#pragma unroll
      for (int t = 0; t < 9; t++) f[s][6 + t] = fp[9 + t];
      const int n = posNode[p0 + pos];
      nd[s] = n;
      v[s][0] = r[3 * (size_t)n]; v[s][1] = r[3 * (size_t)n + 1]; v[s][2] = r[3 * (size_t)n + 2];
    } else {
#pragma unroll
      for (int t = 0; t < 15; t++) f[s][t] = 0;
      v[s][0] = v[s][1] = v[s][2] = 0;
    }
  }
  // forward: y = L_pp^-1 (r - L_p,p-1 y_prev); f[0..5] = (1/l00, 1/l11, l10, 1/l22, l20, l21), f[6..14] = L_p,p-1
  T y0 = 0, y1 = 0, y2 = 0;
#pragma unroll
  for (int s = 0; s < CS_MAXS; s++) {
    if (32 * s >= len) break;
    for (int l = 0; l < 32; l++) {
      const int pos = 32 * s + l;
      if (pos >= len) break;
      if (lane == l) {
        T b0 = v[s][0], b1 = v[s][1], b2 = v[s][2];
        if (pos > 0) {
          b0 -= f[s][6] * y0 + f[s][7] * y1 + f[s][8] * y2;
          b1 -= f[s][9] * y0 + f[s][10] * y1 + f[s][11] * y2;
          b2 -= f[s][12] * y0 + f[s][13] * y1 + f[s][14] * y2;
        }
        const T n0 = b0 * f[s][0];
        const T n1 = (b1 - f[s][2] * n0) * f[s][1];
        const T n2 = (b2 - f[s][4] * n0 - f[s][5] * n1) * f[s][3];
        v[s][0] = n0; v[s][1] = n1; v[s][2] = n2;
        y0 = n0; y1 = n1; y2 = n2;
      }
      y0 = __shfl_sync(0xffffffffu, y0, l);
      y1 = __shfl_sync(0xffffffffu, y1, l);
      y2 = __shfl_sync(0xffffffffu, y2, l);
    }
  }
  // backward: z = L_pp^-T (y - L_p+1,p^T z_next), the product with L_p+1,p formed by the next position's lane
  T t0 = 0, t1 = 0, t2 = 0;
#pragma unroll
  for (int s = CS_MAXS - 1; s >= 0; s--) {
    if (32 * s >= len) continue;
    for (int l = 31; l >= 0; l--) {
      const int pos = 32 * s + l;
      if (pos >= len) continue;
      if (lane == l) {
        T b0 = v[s][0], b1 = v[s][1], b2 = v[s][2];
        if (pos + 1 < len) { b0 -= t0; b1 -= t1; b2 -= t2; }
        const T z2 = b2 * f[s][3];
        const T z1 = (b1 - f[s][5] * z2) * f[s][1];
        const T z0 = (b0 - f[s][2] * z1 - f[s][4] * z2) * f[s][0];
        v[s][0] = z0; v[s][1] = z1; v[s][2] = z2;
        t0 = f[s][6] * z0 + f[s][9] * z1 + f[s][12] * z2;
        t1 = f[s][7] * z0 + f[s][10] * z1 + f[s][13] * z2;
        t2 = f[s][8] * z0 + f[s][11] * z1 + f[s][14] * z2;
      }
      t0 = __shfl_sync(0xffffffffu, t0, l);
      t1 = __shfl_sync(0xffffffffu, t1, l);
      t2 = __shfl_sync(0xffffffffu, t2, l);
    }
  }
#pragma unroll
  for (int s = 0; s < CS_MAXS; s++) {
    if (nd[s] < 0) continue;
    const size_t o = 3 * (size_t)nd[s];
    if (zeroGuess) { x[o] = v[s][0]; x[o + 1] = v[s][1]; x[o + 2] = v[s][2]; }
    else { x[o] += v[s][0]; x[o + 1] += v[s][1]; x[o + 2] += v[s][2]; }
  }
}

MfDims apply_dims(const Context& c, bool fp64) {
  MfDims d;
  d.nx = c.nx; d.ny = c.ny; d.nz = c.nz;
  d.tilesI = (c.nx + MF_TI - 1) / MF_TI;
  d.tilesJ = (c.ny + MF_TJ - 1) / MF_TJ;
  const int maxKs = fp64 ? 8 : 16;
  d.slabs = (c.nz + maxKs - 1) / maxKs;
  d.ks = (c.nz + d.slabs - 1) / d.slabs;
  return d;
}

template <class T, bool RES>
void mf_apply(Context& c, const T* ccK, const T* gs, const T* os, const T* cd, const T* x, const T* b, T* y) {
  const MfDims d = apply_dims(c, sizeof(T) == 8);
  const size_t smem = mf_apply_smem<T>(d.ks);
  if (smem > 48 * 1024) TM_CUDA_CHECK(cudaFuncSetAttribute(k_mf_apply<T, RES>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  k_mf_apply<T, RES><<<d.tilesI * d.tilesJ * d.slabs, MF_THREADS, smem, c.stream>>>(d, c.d_nodeId.p, c.d_cellCls.p, ccK, gs, os, cd, x, b, y);
  note_launch();
  TM_CUDA_CHECK(cudaGetLastError());
}

}  // namespace

// cell classes of the mesh at a stage: (class, scale) of each of the cell's elements, scale = eScale
// (times 1e-6 before the element's group is born, 09-assembly.js:401-403)
void mf_build_cells(Context& c, int stage) {
  if (c.mfStage == stage && c.mfBuilt && c.mfModule == c.moduleStage) return;
  const int ncy = c.ny - 1, ncz = c.nz - 1;
  const size_t ncells = (size_t)(c.nx - 1) * ncy * ncz;
  std::map<std::tuple<int, double, int, double>, int> key;
  std::vector<uint16_t> cellCls(ncells, MF_NONE);
  std::vector<int> info;
  std::vector<double> scale;
  bool ok = true;
  for (size_t cell = 0; cell < ncells && ok; cell++) {
    int cl[2] = {-1, -1};
    double sc[2] = {0, 0};
    int q = 0;
    for (int e2 = 0; e2 < 2; e2++) {
      const int e = c.cellElems[2 * cell + e2];
      if (e < 0) continue;
      const bool born = c.groupStage[c.eGroup[e]] <= stage;
      if (c.moduleStage && !born) continue;   // module stages assemble the born parts only
      cl[q] = c.eClass[e];
      sc[q] = c.eScale[e] * (born ? 1.0 : 1e-6);
      q++;
    }
    if (!q) continue;
    auto t = std::make_tuple(cl[0], sc[0], cl[1], sc[1]);
    auto it = key.find(t);
    int id;
    if (it == key.end()) {
      id = (int)key.size();
      if (id >= MF_MAX_CC) { ok = false; break; }
      key.emplace(t, id);
      info.push_back(cl[0]); info.push_back(cl[1]);
      scale.push_back(sc[0]); scale.push_back(sc[1]);
    } else {
      id = it->second;
    }
    cellCls[cell] = (uint16_t)id;
  }
  int smemMax = 0;
  TM_CUDA_CHECK(cudaDeviceGetAttribute(&smemMax, cudaDevAttrMaxSharedMemoryPerBlockOptin, c.dev));
  c.mfBuilt = true;
  c.mfStage = stage;
  c.mfModule = c.moduleStage;
  // the colour sweep stages whole node columns: meshes with too many node planes keep the stencil
  c.mfAvailable = ok && !key.empty() && TM_MATRIX_FREE && mf_sweep_smem(c.nz) <= (size_t)smemMax &&
                  mf_apply_smem<double>(apply_dims(c, true).ks) <= (size_t)smemMax && c.maxColLen <= 32 * CS_MAXS;
  if (!c.mfAvailable) return;
  c.ncc = (int)key.size();
  cudaStream_t st = c.stream;
  c.d_cellCls.upload(cellCls, st);
  c.d_ccInfo.upload(info, st);
  c.d_ccScale.upload(scale, st);
  c.d_ccK.alloc((size_t)c.ncc * 576);
  c.d_ccK32.alloc((size_t)c.ncc * 576);
  if (!c.d_nodeId.p) c.d_nodeId.upload(c.nodeId, st);
  if (!c.d_colP0.p) {
    std::vector<int> p0((size_t)c.nx * c.ny, -1);
    for (int col = 0; col < c.nx * c.ny; col++)
      if (c.colStart[col + 1] > c.colStart[col]) p0[col] = c.pos[c.colStart[col]];
    c.d_colP0.upload(p0, st);
  }
}

void launch_mf_combine(Context& c) {
  if (!c.mfAvailable) return;
  k_cc_combine<<<c.ncc, 128, 0, c.stream>>>(c.ncc, c.d_ccInfo.p, c.d_ccScale.p, c.d_clsKc.p, c.d_ccK.p, c.d_ccK32.p);
  note_launch();
  TM_CUDA_CHECK(cudaGetLastError());
}

void launch_mf_scales(Context& c, bool scaled) {
  if (!c.mf) return;
  const size_t n = 3 * (size_t)c.nn;
  for (auto* v : {&c.d_gs, &c.d_os, &c.d_cd}) v->alloc(n);
  for (auto* v : {&c.d_gs32, &c.d_os32, &c.d_cd32}) v->alloc(n);
  k_mf_scales<<<grid_for(n, 256), 256, 0, c.stream>>>(c.nn, c.nnp, c.d_pos.p, c.d_isC.p, scaled ? c.d_s.p : nullptr, c.d_val.p, c.d_gs.p,
                                                     c.d_os.p, c.d_cd.p, c.d_gs32.p, c.d_os32.p, c.d_cd32.p);
  note_launch();
  TM_CUDA_CHECK(cudaGetLastError());
}

void launch_mf_apply(Context& c, const double* x, double* y, const double* b) {
  if (b) mf_apply<double, true>(c, c.d_ccK.p, c.d_gs.p, c.d_os.p, c.d_cd.p, x, b, y);
  else mf_apply<double, false>(c, c.d_ccK.p, c.d_gs.p, c.d_os.p, c.d_cd.p, x, nullptr, y);
}

void launch_mf_apply32(Context& c, const float* x, float* y, const float* b) {
  if (b) mf_apply<float, true>(c, c.d_ccK32.p, c.d_gs32.p, c.d_os32.p, c.d_cd32.p, x, b, y);
  else mf_apply<float, false>(c, c.d_ccK32.p, c.d_gs32.p, c.d_os32.p, c.d_cd32.p, x, nullptr, y);
}

size_t mf_sweep_smem(int nz) { return std::max(mf_resid_smem<float>(nz), mf_resid_smem<double>(nz)); }

namespace {
// one colour of the level-0 sweep: the colour's residual rows (not on the cycle's first sweep,
// whose residual is b), then a warp per column solves and updates x
template <class T>
void mf_sweep(Context& c, int col, int zeroGuess, const T* ccK, const T* gs, const T* os, const T* cd, const T* F, const T* b, T* x,
              T* res) {
  MfColDims d;
  d.nx = c.nx; d.ny = c.ny; d.nz = c.nz;
  d.pi = col >> 1; d.pj = col & 1;
  d.rows = (c.nx - d.pi + 1) / 2;
  d.cols = (c.ny - d.pj + 1) / 2;
  if (d.rows <= 0 || d.cols <= 0 || !c.colorCount[col]) return;
  d.tilesJ = (d.cols + RS_SC - 1) / RS_SC;
  if (!zeroGuess) {
    const size_t smem = mf_resid_smem<T>(c.nz);
    if (smem > 48 * 1024) TM_CUDA_CHECK(cudaFuncSetAttribute(k_mf_resid<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k_mf_resid<T><<<d.rows * d.tilesJ, RS_THREADS, smem, c.stream>>>(d, c.d_nodeId.p, c.d_cellCls.p, ccK, gs, os, cd, b, x, res);
    note_launch();
  }
  const int ncols = c.colorCount[col];
  k_col_solve<T><<<grid_for((size_t)ncols * 32, 256), 256, 0, c.stream>>>(ncols, c.d_colPos[col].p, c.d_posNode.p, F, zeroGuess ? b : res,
                                                                         x, zeroGuess);
  note_launch();
  TM_CUDA_CHECK(cudaGetLastError());
}
}  // namespace

void launch_mf_sweep32(Context& c, int col, int zeroGuess, const float* b, float* x) {
  mf_sweep<float>(c, col, zeroGuess, c.d_ccK32.p, c.d_gs32.p, c.d_os32.p, c.d_cd32.p, c.d_F32.p, b, x, c.d_res0_32.p);
}

void launch_mf_sweep64(Context& c, int col, int zeroGuess, const double* b, double* x) {
  mf_sweep<double>(c, col, zeroGuess, c.d_ccK.p, c.d_gs.p, c.d_os.p, c.d_cd.p, c.d_F.p, b, x, c.d_res0.p);
}

}  // namespace tmg
