// Coarse-level set-up of the multigrid preconditioner: the Galerkin coarse operators and the
// coarsest-level direct solver.
//
// Galerkin products (galerkinProduct, src/core/10-solver.js:193-245): coarse block (I, J) is the
// sum of W_i^T K_ij W_j over the fine couplings (i, j) with i under I and j under J. The
// summands of every coarse block are listed once per mesh; a warp sums one block, its lanes
// taking (summand, output column) pairs, five summands at a time, and the five partial columns
// are added in a fixed order (the result does not depend on scheduling).
//
// Coarsest-level direct solver: the banded Cholesky factor of the coarsest shell operator
// (factorCoarsest, src/core/10-solver.js:562-600) and, from it, the explicit inverse that the
// V-cycle applies as one dense product (the reference's solveCoarsest runs the two banded
// substitutions on every cycle instead; both give A^-1 b).
//
// Band layout: row i holds K[i][k] for k in [i-bw, i] at A[i*w + (k - i + bw)], w = bw + 1.
//
// Factor: right-looking blocked Cholesky in steps of CN columns, one launch per step (each launched
// with a programmatic dependency on the previous one, so its launch overlaps that step). A step's
// CTAs each own one CN x CN tile of the trailing window (the rows within bw of the step's
// columns); every CTA factors the step's diagonal block itself, solves the panel rows of its two
// row tiles and subtracts their product from its tile, so no CTA waits on another inside a step;
// CTA 0 also forms the inverse of the diagonal block, in the registers of the warp that factored
// it. The Schur complement stays in the working band; the factor goes to a second band.
//
// Inverse: CTA per pair of groups of NR unit vectors e_j (pairs g, G-1-g balance the work); the
// staged kernel reads each block step's band rows (of L, and of a transposed copy for the
// backward pass) from shared memory filled by cp.async one step ahead. A
// group's forward substitution starts at its first column's block (L^-1 e_j vanishes above j);
// every block of CN rows is one product with the preceding bw rows followed by one product with
// the inverse of the diagonal block, so there is no serial row loop. The backward substitution
// stops at the same block: the inverse is symmetric, so the entries above the diagonal of column
// j come from the columns before it, and each entry is written once (by the solve of the smaller
// of its two indices) on both sides of the diagonal.
#include <cuda_runtime.h>

#include <algorithm>

#include "tm_internal.h"
#include "tm_pdl.cuh"

namespace tmg {

namespace {

constexpr int CN = 32;          // block size of the blocked factor
constexpr int CN_LD = CN + 1;   // padded shared-memory row
constexpr int CHOL_THREADS = 256;

inline int grid_for(size_t n, int block) { return (int)((n + block - 1) / block); }

__device__ __forceinline__ double warp_sum(double v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// ---- Galerkin products ---------------------------------------------------------------------

// galerkinProduct 0 -> 1: summands W_i^T K_ij W_j with 3x3 K_ij (slot s of position ps) and the
// 3x6 weights of the nodes i and j (shellWeights, 10-solver.js:337-353); nn is the row stride of
// the slot-major arrays
__global__ void __launch_bounds__(128) k_galerkin01(int nblk, int nn, const int* __restrict__ start, const int* __restrict__ list,
                                                    const int* __restrict__ posNode, const int* __restrict__ nbr,
                                                    const double* __restrict__ val, const double* __restrict__ W,
                                                    double* __restrict__ out) {
  __shared__ double red[4][5][36];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int g = blockIdx.x * 4 + warp;
  if (g >= nblk) return;
  const int sub = lane / 6, c = lane % 6;
  double acc[6] = {0, 0, 0, 0, 0, 0};
  if (sub < 5) {
    for (int t = start[g] + sub; t < start[g + 1]; t += 5) {
      const int code = list[t];
      const int ps = code / NSLOT, s = code - NSLOT * ps;
      const size_t i = posNode[ps], j = nbr[(size_t)s * nn + ps];
      const double* v = val + (size_t)s * 9 * nn + ps;
      const double* Wi = W + 18 * i;
      const double* Wj = W + 18 * j;
      const double w0 = Wj[c], w1 = Wj[6 + c], w2 = Wj[12 + c];
      const double T0 = v[0] * w0 + v[(size_t)nn] * w1 + v[2 * (size_t)nn] * w2;
      const double T1 = v[3 * (size_t)nn] * w0 + v[4 * (size_t)nn] * w1 + v[5 * (size_t)nn] * w2;
      const double T2 = v[6 * (size_t)nn] * w0 + v[7 * (size_t)nn] * w1 + v[8 * (size_t)nn] * w2;
#pragma unroll
      for (int a = 0; a < 6; a++) acc[a] += Wi[a] * T0 + Wi[6 + a] * T1 + Wi[12 + a] * T2;
    }
#pragma unroll
    for (int a = 0; a < 6; a++) red[warp][sub][a * 6 + c] = acc[a];
  }
  __syncwarp();
  for (int e = lane; e < 36; e += 32)
    out[36 * (size_t)g + e] = (((red[warp][0][e] + red[warp][1][e]) + red[warp][2][e]) + red[warp][3][e]) + red[warp][4][e];
}

// galerkinProduct between shell levels: summands W1^T K W2 with 6x6 fine blocks and 6x6 weights
__global__ void __launch_bounds__(128) k_galerkin_shell(int nblk, const int* __restrict__ start, const int* __restrict__ list,
                                                        const double* __restrict__ fVal, const double* __restrict__ W,
                                                        double* __restrict__ out) {
  __shared__ double red[4][5][36];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int g = blockIdx.x * 4 + warp;
  if (g >= nblk) return;
  const int sub = lane / 6, c = lane % 6;
  double acc[6] = {0, 0, 0, 0, 0, 0};
  if (sub < 5) {
    for (int t = start[g] + sub; t < start[g + 1]; t += 5) {
      const double* K = fVal + 36 * (size_t)list[3 * (size_t)t];
      const double* W1 = W + 36 * (size_t)list[3 * (size_t)t + 1];
      const double* W2 = W + 36 * (size_t)list[3 * (size_t)t + 2];
      double w2[6];
#pragma unroll
      for (int q = 0; q < 6; q++) w2[q] = W2[q * 6 + c];
      double T[6];
#pragma unroll
      for (int r = 0; r < 6; r++)
        T[r] = K[r * 6] * w2[0] + K[r * 6 + 1] * w2[1] + K[r * 6 + 2] * w2[2] + K[r * 6 + 3] * w2[3] + K[r * 6 + 4] * w2[4] +
               K[r * 6 + 5] * w2[5];
#pragma unroll
      for (int a = 0; a < 6; a++)
        acc[a] += W1[a] * T[0] + W1[6 + a] * T[1] + W1[12 + a] * T[2] + W1[18 + a] * T[3] + W1[24 + a] * T[4] + W1[30 + a] * T[5];
    }
#pragma unroll
    for (int a = 0; a < 6; a++) red[warp][sub][a * 6 + c] = acc[a];
  }
  __syncwarp();
  for (int e = lane; e < 36; e += 32)
    out[36 * (size_t)g + e] = (((red[warp][0][e] + red[warp][1][e]) + red[warp][2][e]) + red[warp][3][e]) + red[warp][4][e];
}

// ---- coarsest level --------------------------------------------------------------------------

// lower triangle of the 6x6 block CSR operator into the band, warp per block row
__global__ void k_band_scatter(int nnb, const int* __restrict__ rowPtr, const int* __restrict__ col, const double* __restrict__ val,
                               int bw, double* __restrict__ A) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int i = blockIdx.x * (blockDim.x >> 5) + warp;
  if (i >= nnb) return;
  const int w = bw + 1, k0 = rowPtr[i], nk = rowPtr[i + 1] - k0;
  for (int t = lane; t < 36 * nk; t += 32) {
    const int k = k0 + t / 36, e = t % 36;
    const int j = col[k];
    if (j > i) continue;
    const int r = 6 * i + e / 6, cc = 6 * j + e % 6;
    if (cc <= r && r - cc <= bw) A[(size_t)r * w + (cc - r + bw)] = val[36 * (size_t)k + e];
  }
}

// pivot floor of factorCoarsest: 1e-12 x the largest |diagonal| (1e-12 for a zero diagonal)
__global__ void k_band_jitter(int n, int bw, const double* __restrict__ A, double* __restrict__ jit) {
  __shared__ double s_red[32];
  const int w = bw + 1;
  double dm = 0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) dm = fmax(dm, fabs(A[(size_t)i * w + bw]));
  for (int o = 16; o > 0; o >>= 1) dm = fmax(dm, __shfl_xor_sync(0xffffffffu, dm, o));
  if ((threadIdx.x & 31) == 0) s_red[threadIdx.x >> 5] = dm;
  __syncthreads();
  if (threadIdx.x == 0) {
    double m = 0;
    for (int q = 0; q < (int)(blockDim.x >> 5); q++) m = fmax(m, s_red[q]);
    jit[0] = 1e-12 * (m != 0 ? m : 1);
  }
}

// one block column jb .. jb+nbk-1 of the blocked band Cholesky (see the file comment). Launched
// with a programmatic dependency on the previous step (its launch overlaps that step); the working
// band is read through L2 after the wait (tm_pdl.cuh).
__global__ void __launch_bounds__(CHOL_THREADS) k_band_chol_step(int n, int bw, int jb, double* __restrict__ A, double* __restrict__ Lb,
                                                                 double* __restrict__ Dinv, const double* __restrict__ jit,
                                                                 int* __restrict__ jitterCount) {
  __shared__ double Ds[CN][CN_LD];
  __shared__ double Pi[CN][CN_LD];
  __shared__ double Pj[CN][CN_LD];
  __shared__ double Dv[CN];   // reciprocals of the factor's diagonal
  __shared__ int s_fix;
  grid_dep_launch();
  grid_dep_wait();
  const int w = bw + 1, tid = threadIdx.x;
  constexpr int nthr = CHOL_THREADS;
  const int nbk = min(CN, n - jb);
  const int i0 = jb + nbk, R = min(n, jb + nbk + bw) - i0;
  int ti = 0, tj = blockIdx.x;
  while (tj > ti) { tj -= ti + 1; ti++; }
  // 1. the diagonal block and its factor (warp 0; the same arithmetic in every CTA)
  for (int e = tid; e < CN * CN; e += nthr) {
    const int r = e / CN, cc = e % CN;
    Ds[r][cc] = (r < nbk && cc <= r && r - cc <= bw) ? __ldcg(A + (size_t)(jb + r) * w + (cc - r + bw)) : 0.0;
  }
  if (tid == 0) s_fix = 0;
  __syncthreads();
  // lane r of warp 0 owns row r of the diagonal block through step 2 (its factor row in a[])
  double a[CN];
  double dv = 0;
  if (tid < 32) {
    // right-looking in registers, lane r owning row r: column j's pivot comes from lane j, the
    // column is scaled by the reciprocal square root, and every later row subtracts its rank-1
    // part with the column entries of the other rows brought by shuffles (no shared-memory
    // round trip and no division on the chain)
    const int lane = tid;
    const double jitter = __ldcg(jit);
    int fixes = 0;
#pragma unroll
    for (int k = 0; k < CN; k++) a[k] = Ds[lane][k];
#pragma unroll
    for (int j = 0; j < CN; j++) {
      if (j >= nbk) break;
      double d = __shfl_sync(0xffffffffu, a[j], j);
      if (!(d > jitter)) { d = fmax(fabs(d), jitter); fixes++; }
      const double inv = rsqrt(d);
      const double l = lane > j ? a[j] * inv : (lane == j ? d * inv : 0.0);
      if (lane >= j) a[j] = l;
      if (lane == j) dv = inv;
#pragma unroll
      for (int k = j + 1; k < CN; k++) {
        const double lk = __shfl_sync(0xffffffffu, l, k);
        if (k <= lane) a[k] -= l * lk;
      }
    }
#pragma unroll
    for (int k = 0; k < CN; k++) Ds[lane][k] = (lane < nbk && k <= lane) ? a[k] : 0.0;
    Dv[lane] = lane < nbk ? dv : 0.0;
    if (lane == 0) s_fix = fixes;
  }
  __syncthreads();
  // 2. panel rows of the tiles ti and tj: first the rows of A (all threads, zero outside the
  //    band and the window), then P[r][k] = (A[g][jb+k] - sum_t<k P[r][t] L[k][t]) / L[k][k],
  //    thread per row (warps 2 and 3), in shared memory. Meanwhile warp 0 of CTA 0 forms the
  //    inverse of the diagonal block from the rows it holds.
  for (int e = tid; e < 2 * CN * CN; e += nthr) {
    const int which = e / (CN * CN), r = (e / CN) % CN, k = e % CN;
    if (which == 1 && ti == tj) continue;
    const int tile = which ? tj : ti;
    const int g = i0 + tile * CN + r, kk = jb + k;
    double v = 0;
    if (tile * CN + r < R && k < nbk && g - kk <= bw) v = __ldcg(A + (size_t)g * w + (kk - g + bw));
    (which ? Pj : Pi)[r][k] = v;
  }
  __syncthreads();
  if (tid >= 64 && tid < 128) {
    // right-looking in registers: P[k] is final once the columns before it are subtracted
    const int which = (tid - 64) >> 5, r = tid & 31;
    const int tile = which ? tj : ti;
    double* P = which ? &Pj[r][0] : &Pi[r][0];
    if (!(which == 1 && ti == tj) && tile * CN + r < R) {
      double p[CN];
#pragma unroll
      for (int k = 0; k < CN; k++) p[k] = k < nbk ? P[k] : 0.0;
#pragma unroll
      for (int k = 0; k < CN; k++) {
        if (k >= nbk) break;
        const double pk = p[k] * Dv[k];
        p[k] = pk;
#pragma unroll
        for (int t = k + 1; t < CN; t++) p[t] -= pk * Ds[t][k];
      }
#pragma unroll
      for (int k = 0; k < CN; k++) if (k < nbk) P[k] = p[k];
    }
  }
  if (blockIdx.x == 0 && tid < 32) {
    // column `lane` of L_D^-1 (lower triangular), right-looking: x starts as e_lane, x[k] is
    // final once scaled by 1/L[k][k], and every later x[t] then subtracts L[t][k] x[k] (a[k] of
    // lane t). Each x[t] thus subtracts its terms in the order k = lane, lane+1, ..., t-1.
    const int lane = tid;
    double xv[CN];
#pragma unroll
    for (int r = 0; r < CN; r++) xv[r] = r == lane ? 1.0 : 0.0;
#pragma unroll
    for (int k = 0; k < CN; k++) {
      if (k >= nbk) break;
      const double xk = xv[k] * __shfl_sync(0xffffffffu, dv, k);
      xv[k] = xk;
#pragma unroll
      for (int t = k + 1; t < CN; t++) xv[t] -= __shfl_sync(0xffffffffu, a[k], t) * xk;
    }
    double* Db = Dinv + (size_t)(jb / CN) * CN * CN;
#pragma unroll
    for (int r = 0; r < CN; r++) Db[r * CN + lane] = (r >= lane && r < nbk) ? xv[r] : 0.0;
  }
  __syncthreads();
  // 3. stores of the factor: panel rows by the diagonal tiles, the diagonal block and the pivot
  //    fixes by CTA 0
  if (ti == tj) {
    for (int e = tid; e < CN * CN; e += nthr) {
      const int r = e / CN, k = e % CN;
      const int g = i0 + ti * CN + r, kk = jb + k;
      if (ti * CN + r < R && k < nbk && g - kk <= bw) Lb[(size_t)g * w + (kk - g + bw)] = Pi[r][k];
    }
  }
  if (blockIdx.x == 0) {
    for (int e = tid; e < CN * CN; e += nthr) {
      const int r = e / CN, cc = e % CN;
      if (r < nbk && cc <= r && r - cc <= bw) Lb[(size_t)(jb + r) * w + (cc - r + bw)] = Ds[r][cc];
    }
    if (tid == 0 && s_fix) atomicAdd(jitterCount, s_fix);
  }
  // 4. trailing update of the tile (ti, tj): thread per column cc and four rows rb + 8q, the four
  //    dot products interleaved (each in the order k = 0 .. nbk-1)
  const double(*PJ)[CN_LD] = (ti == tj) ? Pi : Pj;
  static_assert(CHOL_THREADS == 8 * CN, "four rows per thread");
  {
    const int cc = tid % CN, rb = tid / CN;
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
    for (int k = 0; k < nbk; k++) {
      const double pj = PJ[cc][k];
#pragma unroll
      for (int q = 0; q < 4; q++) acc[q] += Pi[rb + 8 * q][k] * pj;
    }
    const int gk = i0 + tj * CN + cc;
#pragma unroll
    for (int q = 0; q < 4; q++) {
      const int r = rb + 8 * q, gi = i0 + ti * CN + r;
      if (ti * CN + r < R && tj * CN + cc < R && gk <= gi && gi - gk <= bw) {
        double* ap = A + (size_t)gi * w + (gk - gi + bw);
        *ap = __ldcg(ap) - acc[q];
      }
    }
  }
}

// the factor's band transposed: Lt[i*w + d] = L[i+d][i] (d = 0 .. bw; zero past the last row)
__global__ void k_band_transpose(int n, int bw, const double* __restrict__ Lb, double* __restrict__ Lt) {
  const int w = bw + 1;
  const size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (t >= (size_t)n * w) return;
  const int i = (int)(t / w), d = (int)(t % w);
  Lt[t] = i + d < n ? Lb[(size_t)(i + d) * w + (bw - d)] : 0.0;
}

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(gmem) : "memory");
}

// Explicit inverse from the blocked factor with the band rows staged in shared memory. The same
// substitutions as k_band_inverse (forward with L, backward with L^T, groups of NR unit vectors,
// pairs g, G-1-g per CTA), but each block step reads its 32 band rows (of L forward, of L^T
// backward: both contiguous, Lb + r0*w and Lt + r0*w) and the diagonal block's inverse from a
// shared-memory buffer that cp.async filled while the previous block step computed, so the
// substitution chain waits on no L2 round trip. Warp r takes row r of the block, lane q the
// terms k = q (mod 32) of its sums for all NR vectors at once (one band value, NR products), and
// the NR sums are reduced over the warp by a fixed butterfly. The buffers and Y take
// 2 * (32 w + 1024) + (n + 32) NR doubles (the launcher checks the fit).
template <int NR>
__device__ __forceinline__ void warp_sum_n(double (&v)[NR]) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1)
#pragma unroll
    for (int c = 0; c < NR; c++) v[c] += __shfl_xor_sync(0xffffffffu, v[c], o);
}
template <int NR>
__global__ void __launch_bounds__(1024) k_band_inverse_staged(int n, int bw, const double* __restrict__ Lb, const double* __restrict__ Lt,
                                                              const double* __restrict__ Dinv, int ngroups, double* __restrict__ inv) {
  static_assert(NR == 2 || NR == 4, "row of Y loaded as double2 pieces");
  extern __shared__ __align__(16) double sms[];
  const int w = bw + 1, tid = threadIdx.x;
  const size_t bufLen = ((size_t)CN * w + CN * CN + 1) & ~(size_t)1;   // 16-byte multiple
  auto buf = [&](int b) { return sms + (size_t)(b & 1) * bufLen; };
  double* Y = sms + 2 * bufLen;       // n x NR, row-major
  double* Z = Y + (size_t)n * NR;     // CN x NR
  const int r = tid >> 5, q = tid & 31;   // blockDim = 1024: warp per block row, lane per term class
  const int nblk = (n + CN - 1) / CN;
  // block b's band rows (of L or of L^T) and its diagonal inverse into buffer b & 1; every copy is
  // 16 bytes between 16-byte boundaries (row blocks start at multiples of 32 w doubles); the last
  // block's rows are rounded up to 16 bytes, which stays inside the band's allocation padding
  auto stage = [&](int b, const double* band) {
    double* dst = buf(b);
    const int rows = min(CN, n - b * CN);
    const int pieces = (int)(((size_t)rows * w * sizeof(double) + 15) / 16);
    const double* src = band + (size_t)b * CN * w;
    for (int e = tid; e < pieces; e += blockDim.x) cp_async16(dst + 2 * e, src + 2 * e);
    const double* db = Dinv + (size_t)b * CN * CN;
    for (int e = tid; e < CN * CN / 2; e += blockDim.x) cp_async16(dst + (size_t)CN * w + 2 * e, db + 2 * e);
    asm volatile("cp.async.commit_group;\n" ::: "memory");
  };
  auto noStage = [] { asm volatile("cp.async.commit_group;\n" ::: "memory"); };
  auto waitStaged = [] { asm volatile("cp.async.wait_group 1;\n" ::: "memory"); };
  // acc[c] += v * Y[k][c] for the NR vectors (the row of Y as double2 loads)
  auto fmaRow = [&](double (&acc)[NR], double v, int k) {
    const double2* yk = reinterpret_cast<const double2*>(Y + (size_t)k * NR);
#pragma unroll
    for (int h = 0; h < NR / 2; h++) {
      const double2 t = yk[h];
      acc[2 * h] += v * t.x;
      acc[2 * h + 1] += v * t.y;
    }
  };
  for (int pass = 0; pass < 2; pass++) {
    const int g = pass == 0 ? (int)blockIdx.x : ngroups - 1 - (int)blockIdx.x;
    if (pass == 1 && g <= (int)blockIdx.x) break;
    const int j0 = g * NR, nr = min(NR, n - j0);
    const int b0 = j0 / CN, rs = b0 * CN;
    // forward: Y = L^-1 E on rows rs .. n-1
    stage(b0, Lb);
    for (int b = b0; b < nblk; b++) {
      if (b + 1 < nblk) stage(b + 1, Lb); else noStage();
      waitStaged();
      __syncthreads();
      const double* Lr = buf(b);
      const double* Db = Lr + (size_t)CN * w;
      const int r0 = b * CN, nbk = min(CN, n - r0);
      const int gr = r0 + r;
      double acc[NR];
#pragma unroll
      for (int c = 0; c < NR; c++) acc[c] = 0;
      if (r < nbk)
        for (int k = max(rs, gr - bw) + q; k < r0; k += 32) fmaRow(acc, Lr[(size_t)r * w + (k - gr + bw)], k);
      warp_sum_n<NR>(acc);
      if (q < NR) {
        double a = acc[0];
#pragma unroll
        for (int c = 1; c < NR; c++) if (q == c) a = acc[c];
        Z[r * NR + q] = (r < nbk ? ((gr == j0 + q && q < nr) ? 1.0 : 0.0) : 0.0) - a;
      }
      __syncthreads();
      double y[NR];
#pragma unroll
      for (int c = 0; c < NR; c++) y[c] = 0;
      if (r < nbk && q <= r) {
        const double d = Db[r * CN + q];
#pragma unroll
        for (int c = 0; c < NR; c++) y[c] = d * Z[q * NR + c];
      }
      warp_sum_n<NR>(y);
      if (q < NR && r < nbk) {
        double a = y[0];
#pragma unroll
        for (int c = 1; c < NR; c++) if (q == c) a = y[c];
        Y[(size_t)gr * NR + q] = a;
      }
      __syncthreads();   // the buffer is refilled two steps on
    }
    // backward: X = L^-T Y on rows n-1 .. rs (X overwrites Y block by block)
    stage(nblk - 1, Lt);
    for (int b = nblk - 1; b >= b0; b--) {
      if (b - 1 >= b0) stage(b - 1, Lt); else noStage();
      waitStaged();
      __syncthreads();
      const double* Ur = buf(b);
      const double* Db = Ur + (size_t)CN * w;
      const int r0 = b * CN, nbk = min(CN, n - r0);
      const int gr = r0 + r;
      double acc[NR];
#pragma unroll
      for (int c = 0; c < NR; c++) acc[c] = 0;
      if (r < nbk) {
        const int kend = min(n, gr + bw + 1);
        for (int k = r0 + nbk + q; k < kend; k += 32) fmaRow(acc, Ur[(size_t)r * w + (k - gr)], k);
      }
      warp_sum_n<NR>(acc);
      if (q < NR) {
        double a = acc[0];
#pragma unroll
        for (int c = 1; c < NR; c++) if (q == c) a = acc[c];
        Z[r * NR + q] = (r < nbk ? Y[(size_t)gr * NR + q] : 0.0) - a;
      }
      __syncthreads();
      double x[NR];
#pragma unroll
      for (int c = 0; c < NR; c++) x[c] = 0;
      if (r < nbk && q >= r && q < nbk) {
        const double d = Db[q * CN + r];
#pragma unroll
        for (int c = 0; c < NR; c++) x[c] = d * Z[q * NR + c];
      }
      warp_sum_n<NR>(x);
      if (q < NR && r < nbk) {
        double a = x[0];
#pragma unroll
        for (int c = 1; c < NR; c++) if (q == c) a = x[c];
        Y[(size_t)gr * NR + q] = a;
      }
      __syncthreads();
    }
    // rows i >= j of column j = j0 + cc, on both sides of the diagonal
    for (size_t e = tid; e < (size_t)(n - rs) * NR; e += blockDim.x) {
      const int i = rs + (int)(e / NR), cc = (int)(e % NR);
      const int j = j0 + cc;
      if (cc < nr && i >= j) {
        const double v = Y[e + (size_t)rs * NR];
        inv[(size_t)i * n + j] = v;
        inv[(size_t)j * n + i] = v;
      }
    }
    __syncthreads();
  }
}

// explicit inverse from the blocked factor (see the file comment). NR unit vectors per group,
// 32/NR partial sums per output reduced with shuffles over adjacent lanes (fixed order).
template <int NR>
__global__ void __launch_bounds__(1024) k_band_inverse(int n, int bw, const double* __restrict__ Lb, const double* __restrict__ Dinv,
                                                       int ngroups, double* __restrict__ inv) {
  constexpr int S = 32 / NR;          // partial sums per output
  extern __shared__ double smi[];
  double* Y = smi;                    // n x NR, row-major
  double* Z = smi + (size_t)n * NR;   // CN x NR
  const int w = bw + 1, tid = threadIdx.x;
  const int o = tid / S, part = tid % S;   // output (r, c) and its part
  const int r = o / NR, c = o % NR;        // blockDim = CN * NR * S = 1024
  const int nblk = (n + CN - 1) / CN;
  for (int pass = 0; pass < 2; pass++) {
    const int g = pass == 0 ? (int)blockIdx.x : ngroups - 1 - (int)blockIdx.x;
    if (pass == 1 && g <= (int)blockIdx.x) break;
    const int j0 = g * NR, nr = min(NR, n - j0);
    const int b0 = j0 / CN, rs = b0 * CN;
    // forward: Y = L^-1 E on rows rs .. n-1
    for (int b = b0; b < nblk; b++) {
      const int r0 = b * CN, nbk = min(CN, n - r0);
      double s = 0;
      if (r < nbk) {
        const int gr = r0 + r;
        const int kbeg = max(rs, gr - bw);
        for (int k = kbeg + part; k < r0; k += S) s += Lb[(size_t)gr * w + (k - gr + bw)] * Y[(size_t)k * NR + c];
      }
#pragma unroll
      for (int q = S / 2; q > 0; q >>= 1) s += __shfl_down_sync(0xffffffffu, s, q, S);
      if (part == 0) Z[r * NR + c] = (r < nbk ? ((r0 + r == j0 + c && c < nr) ? 1.0 : 0.0) : 0.0) - s;
      __syncthreads();
      const double* Db = Dinv + (size_t)b * CN * CN;
      double y = 0;
      if (r < nbk)
        for (int t = part; t <= r; t += S) y += Db[r * CN + t] * Z[t * NR + c];
#pragma unroll
      for (int q = S / 2; q > 0; q >>= 1) y += __shfl_down_sync(0xffffffffu, y, q, S);
      if (part == 0 && r < nbk) Y[(size_t)(r0 + r) * NR + c] = y;
      __syncthreads();
    }
    // backward: X = L^-T Y on rows n-1 .. rs (X overwrites Y block by block)
    for (int b = nblk - 1; b >= b0; b--) {
      const int r0 = b * CN, nbk = min(CN, n - r0);
      double s = 0;
      if (r < nbk) {
        const int gr = r0 + r;
        const int kend = min(n, gr + bw + 1);
        for (int k = r0 + nbk + part; k < kend; k += S) s += Lb[(size_t)k * w + (gr - k + bw)] * Y[(size_t)k * NR + c];
      }
#pragma unroll
      for (int q = S / 2; q > 0; q >>= 1) s += __shfl_down_sync(0xffffffffu, s, q, S);
      if (part == 0) Z[r * NR + c] = (r < nbk ? Y[(size_t)(r0 + r) * NR + c] : 0.0) - s;
      __syncthreads();
      const double* Db = Dinv + (size_t)b * CN * CN;
      double x = 0;
      if (r < nbk)
        for (int t = r + part; t < nbk; t += S) x += Db[t * CN + r] * Z[t * NR + c];
#pragma unroll
      for (int q = S / 2; q > 0; q >>= 1) x += __shfl_down_sync(0xffffffffu, x, q, S);
      if (part == 0 && r < nbk) Y[(size_t)(r0 + r) * NR + c] = x;
      __syncthreads();
    }
    // rows i >= j of column j = j0 + cc, on both sides of the diagonal
    for (size_t e = tid; e < (size_t)(n - rs) * NR; e += blockDim.x) {
      const int i = rs + (int)(e / NR), cc = (int)(e % NR);
      const int j = j0 + cc;
      if (cc < nr && i >= j) {
        const double v = Y[e + (size_t)rs * NR];
        inv[(size_t)i * n + j] = v;
        inv[(size_t)j * n + i] = v;
      }
    }
    __syncthreads();
  }
}

// general fallback for a coarsest level too large for the shared-memory work vectors: warp per
// unit vector e_c, the result row c (the inverse is symmetric) doubling as the work vector
__global__ void k_band_inverse_warp(int n, int bw, const double* __restrict__ A, double* __restrict__ inv) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int c = blockIdx.x * (blockDim.x >> 5) + warp;
  if (c >= n) return;
  const int w = bw + 1;
  double* y = inv + (size_t)c * n;
  for (int i = lane; i < c; i += 32) y[i] = 0;
  __syncwarp();
  for (int i = c; i < n; i++) {
    double ss = 0;
    for (int k = max(c, i - bw) + lane; k < i; k += 32) ss += A[(size_t)i * w + (k - i + bw)] * y[k];
    ss = warp_sum(ss);
    if (lane == 0) y[i] = ((i == c ? 1.0 : 0.0) - ss) / A[(size_t)i * w + bw];
    __syncwarp();
  }
  for (int i = n - 1; i >= 0; i--) {
    double ss = 0;
    const int kend = min(n, i + bw + 1);
    for (int k = i + 1 + lane; k < kend; k += 32) ss += A[(size_t)k * w + (i - k + bw)] * y[k];
    ss = warp_sum(ss);
    if (lane == 0) y[i] = (y[i] - ss) / A[(size_t)i * w + bw];
    __syncwarp();
  }
}

template <int NR>
bool try_band_inverse_staged(Context& c, ShellLevel& L) {
  const int n = L.denseN, bw = L.bandBw, w = bw + 1;
  const size_t bufLen = ((size_t)CN * w + CN * CN + 1) & ~(size_t)1;
  const size_t smem = (2 * bufLen + (size_t)(n + CN) * NR) * sizeof(double);
  int smemMax = 0;
  TM_CUDA_CHECK(cudaDeviceGetAttribute(&smemMax, cudaDevAttrMaxSharedMemoryPerBlockOptin, c.dev));
  if (smem > (size_t)smemMax) return false;
  L.d_bandLt.alloc((size_t)n * w);
  k_band_transpose<<<grid_for((size_t)n * w, 256), 256, 0, c.stream>>>(n, bw, L.d_bandL.p, L.d_bandLt.p);
  TM_CUDA_CHECK(cudaFuncSetAttribute(k_band_inverse_staged<NR>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const int ngroups = (n + NR - 1) / NR;
  k_band_inverse_staged<NR><<<(ngroups + 1) / 2, 1024, smem, c.stream>>>(n, bw, L.d_bandL.p, L.d_bandLt.p, L.d_dinv.p, ngroups, L.d_inv.p);
  note_launch(2);
  return true;
}

template <int NR>
bool try_band_inverse(Context& c, ShellLevel& L) {
  const int n = L.denseN;
  const size_t smem = ((size_t)n * NR + (size_t)CN * NR) * sizeof(double);
  if (smem > 200 * 1024) return false;
  TM_CUDA_CHECK(cudaFuncSetAttribute(k_band_inverse<NR>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const int ngroups = (n + NR - 1) / NR;
  k_band_inverse<NR><<<(ngroups + 1) / 2, 1024, smem, c.stream>>>(n, L.bandBw, L.d_bandL.p, L.d_dinv.p, ngroups, L.d_inv.p);
  note_launch();
  return true;
}

}  // namespace

void launch_galerkin01(Context& c) {
  ShellLevel& L1 = *c.shells[0];
  note_launch();
  TimedLaunch tl(c, K_GALERKIN01);
  k_galerkin01<<<grid_for(L1.nb, 4), 128, 0, c.stream>>>(L1.nb, c.nnp, c.d_g01Start.p, c.d_g01List.p, c.d_posNode.p, c.d_nbr.p, c.d_val.p,
                                                        c.d_W01.p, L1.d_val.p);
  TM_CUDA_CHECK(cudaGetLastError());
}

void launch_galerkin_shell(Context& c, int l) {
  ShellLevel& F = *c.shells[l];
  ShellLevel& C = *c.shells[l + 1];
  note_launch();
  k_galerkin_shell<<<grid_for(C.nb, 4), 128, 0, c.stream>>>(C.nb, C.d_galStart.p, C.d_galList.p, F.d_val.p, F.d_prolW.p, C.d_val.p);
  TM_CUDA_CHECK(cudaGetLastError());
}

void launch_factor_coarsest(Context& c, ShellLevel& L) {
  const int n = L.denseN, bw = L.bandBw, w = bw + 1;
  if (n <= 0) return;
  L.d_bandL.alloc((size_t)n * w);
  L.d_dinv.alloc((size_t)((n + CN - 1) / CN) * CN * CN);
  L.d_jit.alloc(1);
  TM_CUDA_CHECK(cudaMemsetAsync(L.d_band.p, 0, (size_t)n * w * sizeof(double), c.stream));
  TM_CUDA_CHECK(cudaMemsetAsync(L.d_bandL.p, 0, (size_t)n * w * sizeof(double), c.stream));
  k_band_scatter<<<grid_for(L.nn, 4), 128, 0, c.stream>>>(L.nn, L.d_rowPtr.p, L.d_col.p, L.d_val.p, bw, L.d_band.p);
  k_band_jitter<<<1, 1024, 0, c.stream>>>(n, bw, L.d_band.p, L.d_jit.p);
  note_launch(2);
  for (int jb = 0; jb < n; jb += CN) {
    const int nbk = std::min(CN, n - jb);
    const int R = std::min(n, jb + nbk + bw) - (jb + nbk);
    const int T = (R + CN - 1) / CN;
    const int ncta = std::max(1, T * (T + 1) / 2);
    launch_pdl(k_band_chol_step, ncta, CHOL_THREADS, 0, c.stream, n, bw, jb, L.d_band.p, L.d_bandL.p, L.d_dinv.p, (const double*)L.d_jit.p,
               c.d_jitter.p);
    note_launch();
  }
  TM_CUDA_CHECK(cudaGetLastError());
  if (!try_band_inverse_staged<4>(c, L) && !try_band_inverse_staged<2>(c, L) && !try_band_inverse<8>(c, L) && !try_band_inverse<4>(c, L) &&
      !try_band_inverse<2>(c, L) && !try_band_inverse<1>(c, L)) {
    k_band_inverse_warp<<<grid_for(n, 4), 128, 0, c.stream>>>(n, bw, L.d_bandL.p, L.d_inv.p);
    note_launch();
  }
  TM_CUDA_CHECK(cudaGetLastError());
}

}  // namespace tmg
