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
// xs: staged gs*x, 3 values per node, node (ii, jj, kk) at ((kk*PI + ii)*PJ + jj)*3; cls: staged cell
// classes, cell (ci, cj, ck) at (ck*CI + ci)*CJ + cj, where the node's own cell-corner indices are
// (ii-1, jj-1, kk-1) .. (ii, jj, kk) in staged-cell coordinates shifted by one (cell (ii-1+a) is staged
// at ii-1+a + co, co = the cell-coordinate offset of the stage)
template <class T>
struct KRow;
template <>
struct KRow<float> {
  // 24 values of row r of cell class cc
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

// acc += (K x) rows of the node at staged node coordinates (ii, jj, kk); staged cell (ci, cj, ck) of
// the cell whose corner at offsets (1-a, 1-b, 1-c) is this node sits at (ii-1+a+cio, jj-1+b+cjo, kk-1+c+cko)
template <class T, int PI, int PJ, int CI, int CJ>
__device__ __forceinline__ void node_row(const T* __restrict__ xs, const uint16_t* __restrict__ cls, const T* __restrict__ ccK, int ii, int jj,
                                         int kk, int ci0, int cj0, int ck0, T (&acc)[3]) {
#pragma unroll
  for (int c = 0; c < 2; c++)
#pragma unroll
    for (int b = 0; b < 2; b++)
#pragma unroll
      for (int a = 0; a < 2; a++) {
        const int cc = cls[((ck0 + c) * CI + ci0 + a) * CJ + cj0 + b];
        if (cc == MF_NONE) continue;
        // the cell's 8 nodes, gathered in the local order of the element matrix
        T xv[24];
#pragma unroll
        for (int M = 0; M < 8; M++) {
          const T* xp = xs + (((kk - 1 + c + loc_c(M)) * PI + ii - 1 + a + loc_a(M)) * PJ + jj - 1 + b + loc_b(M)) * 3;
          xv[3 * M] = xp[0]; xv[3 * M + 1] = xp[1]; xv[3 * M + 2] = xp[2];
        }
        const int Lrow = loc_of(1 - a, 1 - b, 1 - c);
        const T* K = ccK + (size_t)cc * 576 + 3 * Lrow * 24;
#pragma unroll
        for (int p = 0; p < 3; p++) {
          T k[24];
          KRow<T>::load(K + 24 * p, k);
          T s = 0;
#pragma unroll
          for (int q = 0; q < 24; q++) s += k[q] * xv[q];
          acc[p] += s;
        }
      }
}

// ---- staging of a box of nodes and cells into shared memory -----------------------------------------
// Items are walked with the node planes fastest (consecutive node ids of a column, coalesced). Each
// thread keeps SB items in flight: first all their node ids, then all their x and gs, so a thread
// waits for two rounds of loads per SB items instead of two per item.
constexpr int SB = 8;

// gs*x of the box of PI x PJ node columns from (i0, j0), planes k0 .. k0+np-1, into
// xs[((kk*PI + ii)*PJ + jj)*3 ..] (zero outside the mesh and where no node exists); when ids is not
// null, the node ids (-1 for none) into ids[(kk*PI + ii)*PJ + jj]
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
      T* dst = xs + 3 * (size_t)at;
      dst[0] = v[u][0]; dst[1] = v[u][1]; dst[2] = v[u][2];
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
constexpr int MF_TI = 8, MF_TJ = 8;
constexpr int MF_PI = MF_TI + 2, MF_PJ = MF_TJ + 2;       // staged node columns (one halo column each side)
constexpr int MF_CI = MF_TI + 1, MF_CJ = MF_TJ + 1;       // staged cell columns
constexpr int MF_THREADS = 256;

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
  const size_t nodes = (size_t)np * MF_PI * MF_PJ;
  T* xs = reinterpret_cast<T*>(smraw);
  int* ids = reinterpret_cast<int*>(xs + nodes * 3);
  uint16_t* cls = reinterpret_cast<uint16_t*>(ids + nodes);
  int blk = blockIdx.x;
  const int slab = blk % d.slabs; blk /= d.slabs;
  const int tj = blk % d.tilesJ, ti = blk / d.tilesJ;
  const int i0 = ti * MF_TI, j0 = tj * MF_TJ, k0 = slab * ks;
  // gs*x and the node ids of the tile's node columns plus one halo column and plane on every side,
  // and the cell classes of cells (i0-1 .. i0+TI-1) x (j0-1 ..) x (k0-1 .. k0+ks-1)
  stage_nodes<T, MF_PI, MF_PJ>(d.nx, d.ny, d.nz, i0 - 1, j0 - 1, k0 - 1, np, nodeId, x, gs, xs, ids);
  stage_cells<MF_CI, MF_CJ>(d.nx, d.ny, d.nz, i0 - 1, j0 - 1, k0 - 1, ks + 1, cellCls, cls);
  __syncthreads();
  // node (i0+ii, j0+jj, k0+kk): a warp takes half a plane of the tile (4 x 8 columns), so that its
  // lanes read the same cell classes (one layer) and the class table loads are warp-uniform
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int ii = (warp & 1) * 4 + (lane >> 3), jj = lane & 7;
  const int i = i0 + ii, j = j0 + jj;
  if (i >= d.nx || j >= d.ny) return;
  for (int kk = warp >> 1; kk < ks; kk += MF_THREADS / 64) {
    const int k = k0 + kk;
    if (k >= d.nz) break;
    const int n = ids[((kk + 1) * MF_PI + ii + 1) * MF_PJ + jj + 1];
    if (n < 0) continue;
    T acc[3] = {0, 0, 0};
    // staged node coordinates of the node: (ii+1, jj+1, kk+1); staged cell coordinates of the cell
    // (i-1+a, j-1+b, k-1+c): (ii+a, jj+b, kk+c)
    node_row<T, MF_PI, MF_PJ, MF_CI, MF_CJ>(xs, cls, ccK, ii + 1, jj + 1, kk + 1, ii, jj, kk, acc);
    const size_t o = 3 * (size_t)n;
#pragma unroll
    for (int p = 0; p < 3; p++) {
      const T g = gs[o + p];
      const T v = g != (T)0 ? os[o + p] * acc[p] : cd[o + p] * x[o + p];
      y[o + p] = RES ? b[o + p] - v : v;
    }
  }
}

// ---- colour sweep: tiles of SR x SC columns of one colour -------------------------------------------
// The tile's columns are (pi + 2 r, pj + 2 c) for r < SR, c < SC (colour rows and columns of the
// tile); their neighbours span 2 SR + 1 x 2 SC + 1 node columns, staged over all node planes. The
// column factors of the tile's columns are copied into shared memory asynchronously while the
// residual rows are computed. FP32: 2 x 8 columns (the 32 lanes of a warp take two planes); FP64:
// 1 x 8 (four planes per warp), which keeps two CTAs per SM.
constexpr int SW_SC = 8;
constexpr int SW_THREADS = 256;
template <class T>
struct SwShape { static constexpr int SR = sizeof(T) == 4 ? 2 : 1; };

struct SwLayout {
  size_t xs, cls, F, r, nid, meta, total;
};
template <class T>
inline SwLayout sw_layout(int nz) {
  constexpr int SR = SwShape<T>::SR, SLOTS = SR * SW_SC;
  constexpr int PI = 2 * SR + 1, PJ = 2 * SW_SC + 1, CI = 2 * SR, CJ = 2 * SW_SC;
  SwLayout L;
  size_t o = 0;
  auto take = [&](size_t bytes) { const size_t at = o; o = (o + bytes + 15) / 16 * 16; return at; };
  // node planes -1 .. nz and cell layers -1 .. nz-1, zero / no class outside the mesh
  L.xs = take((size_t)(nz + 2) * PI * PJ * 3 * sizeof(T));
  L.cls = take((size_t)(nz + 1) * CI * CJ * sizeof(uint16_t));
  L.F = take((size_t)SLOTS * nz * 18 * sizeof(T));
  L.r = take((size_t)SLOTS * nz * 3 * sizeof(T));
  L.nid = take((size_t)SLOTS * nz * sizeof(int));
  L.meta = take((size_t)SLOTS * 2 * sizeof(int));
  L.total = o;
  return L;
}

struct MfSweepDims {
  int nx, ny, nz;
  int pi, pj;          // colour parities
  int rows, cols;      // colour rows / columns of the colour
  int tilesJ;          // tiles along the colour columns
};

__device__ __forceinline__ void cp_async8(void* smem, const void* gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

template <class T>
__global__ void __launch_bounds__(SW_THREADS) k_mf_sweep(MfSweepDims d, SwLayout lay, const int* __restrict__ nodeId,
                                                         const int* __restrict__ colStart, const int* __restrict__ colP0,
                                                         const uint16_t* __restrict__ cellCls, const T* __restrict__ ccK,
                                                         const T* __restrict__ gs, const T* __restrict__ os, const T* __restrict__ cd,
                                                         const T* __restrict__ F, const T* __restrict__ b, T* __restrict__ x,
                                                         int zeroGuess) {
  constexpr int SR = SwShape<T>::SR, SC = SW_SC, SLOTS = SR * SC;
  constexpr int PI = 2 * SR + 1, PJ = 2 * SC + 1, CI = 2 * SR, CJ = 2 * SC;
  constexpr int PLANES_PER_WARP = 32 / SLOTS;
  extern __shared__ __align__(16) unsigned char smraw[];
  T* xs = reinterpret_cast<T*>(smraw + lay.xs);
  uint16_t* cls = reinterpret_cast<uint16_t*>(smraw + lay.cls);
  T* Fs = reinterpret_cast<T*>(smraw + lay.F);
  T* rs = reinterpret_cast<T*>(smraw + lay.r);
  int* nid = reinterpret_cast<int*>(smraw + lay.nid);
  int* meta = reinterpret_cast<int*>(smraw + lay.meta);
  const int nz = d.nz, ncy = d.ny - 1, ncz = d.nz - 1;
  const int tr = blockIdx.x / d.tilesJ, tc = blockIdx.x % d.tilesJ;
  const int iLo = d.pi + 2 * SR * tr - 1, jLo = d.pj + 2 * SC * tc - 1;   // first staged node column
  // the tile's columns: first position and length
  if (threadIdx.x < SLOTS) {
    const int r = threadIdx.x / SC, c = threadIdx.x % SC;
    const int cr = SR * tr + r, ccol = SC * tc + c;
    int p0 = -1, len = 0;
    if (cr < d.rows && ccol < d.cols) {
      const int col = (d.pi + 2 * cr) * d.ny + d.pj + 2 * ccol;
      len = colStart[col + 1] - colStart[col];
      p0 = len > 0 ? colP0[col] : -1;
    }
    meta[2 * threadIdx.x] = p0;
    meta[2 * threadIdx.x + 1] = len;
  }
  __syncthreads();
  // column factors (18 per node, position order) -> Fs[slot][l][18], asynchronously in 8-byte pieces
  for (int s = 0; s < SLOTS; s++) {
    const int p0 = meta[2 * s], len = meta[2 * s + 1];
    if (p0 < 0) continue;
    const unsigned char* src = reinterpret_cast<const unsigned char*>(F + 18 * (size_t)p0);
    unsigned char* dst = reinterpret_cast<unsigned char*>(Fs + (size_t)s * nz * 18);
    const int pieces = (int)(18 * sizeof(T) / 8) * len;
    for (int e = threadIdx.x; e < pieces; e += blockDim.x) cp_async8(dst + 8 * e, src + 8 * e);
  }
  asm volatile("cp.async.commit_group;\n" ::: "memory");
  // the node ids of the tile's columns (-1: none), SB per thread in flight
  for (int t0 = threadIdx.x; t0 < SLOTS * nz; t0 += SB * blockDim.x) {
    int n[SB];
#pragma unroll
    for (int u = 0; u < SB; u++) {
      const int t = t0 + u * blockDim.x;
      n[u] = -1;
      if (t < SLOTS * nz) {
        const int sl = t / nz, k = t % nz;
        if (meta[2 * sl] >= 0) n[u] = nodeId[((size_t)(iLo + 1 + 2 * (sl / SC)) * d.ny + jLo + 1 + 2 * (sl % SC)) * nz + k];
      }
    }
#pragma unroll
    for (int u = 0; u < SB; u++) {
      const int t = t0 + u * blockDim.x;
      if (t < SLOTS * nz) nid[t] = n[u];
    }
  }
  if (!zeroGuess) {
    // node plane k is staged at k+1, cell layer k at k+1
    stage_nodes<T, PI, PJ>(d.nx, d.ny, nz, iLo, jLo, -1, nz + 2, nodeId, x, gs, xs, nullptr);
    stage_cells<CI, CJ>(d.nx, d.ny, nz, iLo, jLo, -1, ncz + 2, cellCls, cls);
  }
  __syncthreads();
  // residual rows r = b - Ks x of the tile's columns: the lanes of a warp take the SLOTS columns at
  // PLANES_PER_WARP consecutive planes
  {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int s = lane % SLOTS;
    const int r = s / SC, c = s % SC;
    const int ii = 1 + 2 * r, jj = 1 + 2 * c;   // staged coordinates of the column
    const int i = iLo + ii, j = jLo + jj;
    const bool colOk = meta[2 * s] >= 0;
    for (int k = PLANES_PER_WARP * warp + lane / SLOTS; k < nz; k += PLANES_PER_WARP * (SW_THREADS / 32)) {
      const int n = colOk ? nid[s * nz + k] : -1;
      if (n < 0) continue;
      const size_t o = 3 * (size_t)n;
      T rv[3] = {b[o], b[o + 1], b[o + 2]};
      if (!zeroGuess) {
        T acc[3] = {0, 0, 0};
        // cell (i-1+a, j-1+b, k-1+c) is staged at (ii-1+a, jj-1+b, k+c); node (i, j, k) at (ii, jj, k+1)
        node_row<T, PI, PJ, CI, CJ>(xs, cls, ccK, ii, jj, k + 1, ii - 1, jj - 1, k, acc);
#pragma unroll
        for (int p = 0; p < 3; p++) {
          const T g = gs[o + p];
          rv[p] -= g != (T)0 ? os[o + p] * acc[p] : cd[o + p] * x[o + p];
        }
      }
      T* rp = rs + ((size_t)s * nz + k) * 3;
      rp[0] = rv[0]; rp[1] = rv[1]; rp[2] = rv[2];
    }
  }
  cp_async_wait_all();
  __syncthreads();
  // block-tridiagonal solve of every column (solveColumn, 10-solver.js:71-104), one thread per column,
  // with the reciprocal pivots stored in the factors' upper slots; absent planes are skipped
  if (threadIdx.x < SLOTS && meta[2 * threadIdx.x] >= 0) {
    const int s = threadIdx.x;
    const T* Fc = Fs + (size_t)s * nz * 18;
    T* rc = rs + (size_t)s * nz * 3;
    const int* nc = nid + s * nz;
    T p0 = 0, p1 = 0, p2 = 0;
    int l = 0;
    for (int k = 0; k < nz; k++) {
      if (nc[k] < 0) continue;
      const T* f = Fc + 18 * l;
      T b0 = rc[3 * k], b1 = rc[3 * k + 1], b2 = rc[3 * k + 2];
      if (l > 0) {
        b0 -= f[9] * p0 + f[10] * p1 + f[11] * p2;
        b1 -= f[12] * p0 + f[13] * p1 + f[14] * p2;
        b2 -= f[15] * p0 + f[16] * p1 + f[17] * p2;
      }
      p0 = b0 * f[1];
      p1 = (b1 - f[3] * p0) * f[2];
      p2 = (b2 - f[6] * p0 - f[7] * p1) * f[5];
      rc[3 * k] = p0; rc[3 * k + 1] = p1; rc[3 * k + 2] = p2;
      l++;
    }
    T q0 = 0, q1 = 0, q2 = 0;
    const T* g = nullptr;
    for (int k = nz - 1; k >= 0; k--) {
      if (nc[k] < 0) continue;
      l--;
      const T* f = Fc + 18 * l;
      T b0 = rc[3 * k], b1 = rc[3 * k + 1], b2 = rc[3 * k + 2];
      if (g) {
        b0 -= g[9] * q0 + g[12] * q1 + g[15] * q2;
        b1 -= g[10] * q0 + g[13] * q1 + g[16] * q2;
        b2 -= g[11] * q0 + g[14] * q1 + g[17] * q2;
      }
      q2 = b2 * f[5];
      q1 = (b1 - f[7] * q2) * f[2];
      q0 = (b0 - f[3] * q1 - f[6] * q2) * f[1];
      rc[3 * k] = q0; rc[3 * k + 1] = q1; rc[3 * k + 2] = q2;
      g = f;
    }
  }
  __syncthreads();
  // x += dx
  for (int t = threadIdx.x; t < SLOTS * nz; t += blockDim.x) {
    const int n = nid[t];
    if (n < 0) continue;
    const T* rp = rs + (size_t)t * 3;
    const size_t o = 3 * (size_t)n;
    if (zeroGuess) { x[o] = rp[0]; x[o + 1] = rp[1]; x[o + 2] = rp[2]; }
    else { x[o] += rp[0]; x[o + 1] += rp[1]; x[o + 2] += rp[2]; }
  }
}

MfDims apply_dims(const Context& c) {
  MfDims d;
  d.nx = c.nx; d.ny = c.ny; d.nz = c.nz;
  d.tilesI = (c.nx + MF_TI - 1) / MF_TI;
  d.tilesJ = (c.ny + MF_TJ - 1) / MF_TJ;
  d.slabs = (c.nz + 15) / 16;
  d.ks = (c.nz + d.slabs - 1) / d.slabs;
  return d;
}

template <class T, bool RES>
void mf_apply(Context& c, const T* ccK, const T* gs, const T* os, const T* cd, const T* x, const T* b, T* y) {
  const MfDims d = apply_dims(c);
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
                  mf_apply_smem<double>(apply_dims(c).ks) <= (size_t)smemMax;
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

size_t mf_sweep_smem(int nz) { return std::max(sw_layout<float>(nz).total, sw_layout<double>(nz).total); }

namespace {
template <class T>
void mf_sweep(Context& c, int col, int zeroGuess, const T* ccK, const T* gs, const T* os, const T* cd, const T* F, const T* b, T* x) {
  constexpr int SR = SwShape<T>::SR;
  MfSweepDims d;
  d.nx = c.nx; d.ny = c.ny; d.nz = c.nz;
  d.pi = col >> 1; d.pj = col & 1;
  d.rows = (c.nx - d.pi + 1) / 2;
  d.cols = (c.ny - d.pj + 1) / 2;
  if (d.rows <= 0 || d.cols <= 0) return;
  d.tilesJ = (d.cols + SW_SC - 1) / SW_SC;
  const int tilesI = (d.rows + SR - 1) / SR;
  const SwLayout lay = sw_layout<T>(c.nz);
  if (lay.total > 48 * 1024) TM_CUDA_CHECK(cudaFuncSetAttribute(k_mf_sweep<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)lay.total));
  k_mf_sweep<T><<<tilesI * d.tilesJ, SW_THREADS, lay.total, c.stream>>>(d, lay, c.d_nodeId.p, c.d_colStart.p, c.d_colP0.p, c.d_cellCls.p,
                                                                      ccK, gs, os, cd, F, b, x, zeroGuess);
  note_launch();
  TM_CUDA_CHECK(cudaGetLastError());
}
}  // namespace

void launch_mf_sweep32(Context& c, int col, int zeroGuess, const float* b, float* x) {
  mf_sweep<float>(c, col, zeroGuess, c.d_ccK32.p, c.d_gs32.p, c.d_os32.p, c.d_cd32.p, c.d_F32.p, b, x);
}

void launch_mf_sweep64(Context& c, int col, int zeroGuess, const double* b, double* x) {
  mf_sweep<double>(c, col, zeroGuess, c.d_ccK.p, c.d_gs.p, c.d_os.p, c.d_cd.p, c.d_F.p, b, x);
}

}  // namespace tmg
