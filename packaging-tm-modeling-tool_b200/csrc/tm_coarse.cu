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
// Factor: right-looking blocked Cholesky in steps of CN columns, one launch per step. A step's
// CTAs each own one CN x CN tile of the trailing window (the rows within bw of the step's
// columns); every CTA factors the step's diagonal block itself, solves the panel rows of its two
// row tiles and subtracts their product from its tile, so no CTA waits on another inside a step.
// The Schur complement stays in the working band; the factor goes to a second band.
//
// Inverse: CTA per pair of groups of NR unit vectors e_j (pairs g, G-1-g balance the work). A
// group's forward substitution starts at its first column's block (L^-1 e_j vanishes above j);
// every block of CN rows is one product with the preceding bw rows followed by one product with
// the inverse of the diagonal block, so there is no serial row loop. The backward substitution
// stops at the same block: the inverse is symmetric, so the entries above the diagonal of column
// j come from the columns before it, and each entry is written once (by the solve of the smaller
// of its two indices) on both sides of the diagonal.
#include <cuda_runtime.h>

#include <algorithm>

#include "tm_internal.h"

namespace tmg {

namespace {

constexpr int CN = 32;          // block size of the blocked factor
constexpr int CN_LD = CN + 1;   // padded shared-memory row

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

// one block column jb .. jb+nbk-1 of the blocked band Cholesky (see the file comment)
__global__ void __launch_bounds__(256) k_band_chol_step(int n, int bw, int jb, double* __restrict__ A, double* __restrict__ Lb,
                                                        double* __restrict__ Dinv, const double* __restrict__ jit,
                                                        int* __restrict__ jitterCount) {
  __shared__ double Ds[CN][CN_LD];
  __shared__ double Pi[CN][CN_LD];
  __shared__ double Pj[CN][CN_LD];
  __shared__ double Dv[CN];   // reciprocals of the factor's diagonal
  __shared__ int s_fix;
  const int w = bw + 1, tid = threadIdx.x, nthr = blockDim.x;
  const int nbk = min(CN, n - jb);
  const int i0 = jb + nbk, R = min(n, jb + nbk + bw) - i0;
  int ti = 0, tj = blockIdx.x;
  while (tj > ti) { tj -= ti + 1; ti++; }
  // 1. the diagonal block and its factor (warp 0; the same arithmetic in every CTA)
  for (int e = tid; e < CN * CN; e += nthr) {
    const int r = e / CN, cc = e % CN;
    Ds[r][cc] = (r < nbk && cc <= r && r - cc <= bw) ? A[(size_t)(jb + r) * w + (cc - r + bw)] : 0.0;
  }
  if (tid == 0) s_fix = 0;
  __syncthreads();
  if (tid < 32) {
    // right-looking in registers, lane r owning row r: column j's pivot comes from lane j, the
    // column is scaled by the reciprocal square root, and every later row subtracts its rank-1
    // part with the column entries of the other rows brought by shuffles (no shared-memory
    // round trip and no division on the chain)
    const int lane = tid;
    const double jitter = jit[0];
    int fixes = 0;
    double a[CN];
#pragma unroll
    for (int k = 0; k < CN; k++) a[k] = Ds[lane][k];
    double dv = 0;
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
  //    thread per row, in shared memory
  for (int e = tid; e < 2 * CN * CN; e += nthr) {
    const int which = e / (CN * CN), r = (e / CN) % CN, k = e % CN;
    if (which == 1 && ti == tj) continue;
    const int tile = which ? tj : ti;
    const int g = i0 + tile * CN + r, kk = jb + k;
    double a = 0;
    if (tile * CN + r < R && k < nbk && g - kk <= bw) a = A[(size_t)g * w + (kk - g + bw)];
    (which ? Pj : Pi)[r][k] = a;
  }
  __syncthreads();
  if (tid < 64) {
    // right-looking in registers: P[k] is final once the columns before it are subtracted
    const int which = tid >> 5, r = tid & 31;
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
  __syncthreads();
  // 3. stores of the factor: panel rows by the diagonal tiles, the diagonal block, its inverse and
  //    the pivot fixes by CTA 0
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
    // column c of the inverse of the diagonal block (lower triangular), thread per column; Pj is
    // free in CTA 0 (its tile pair is (0, 0)) and holds the columns
    if (tid < CN) {
      const int c = tid;
      for (int r = 0; r < CN; r++) {
        double x = 0;
        if (r >= c && r < nbk) {
          double s = (r == c) ? 1.0 : 0.0;
          for (int t = c; t < r; t++) s -= Ds[r][t] * Pj[t][c];
          x = s * Dv[r];
        }
        Pj[r][c] = x;
      }
    }
    __syncthreads();
    double* Db = Dinv + (size_t)(jb / CN) * CN * CN;
    for (int e = tid; e < CN * CN; e += nthr) Db[e] = Pj[e / CN][e % CN];
    if (tid == 0 && s_fix) atomicAdd(jitterCount, s_fix);
  }
  // 4. trailing update of the tile (ti, tj) (CTA 0 reused Pj above; its tile pair reads Pi only)
  const double(*PJ)[CN_LD] = (ti == tj) ? Pi : Pj;
  for (int e = tid; e < CN * CN; e += nthr) {
    const int r = e / CN, cc = e % CN;
    const int gi = i0 + ti * CN + r, gk = i0 + tj * CN + cc;
    if (ti * CN + r < R && tj * CN + cc < R && gk <= gi && gi - gk <= bw) {
      double s = 0;
      for (int k = 0; k < nbk; k++) s += Pi[r][k] * PJ[cc][k];
      A[(size_t)gi * w + (gk - gi + bw)] -= s;
    }
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
    k_band_chol_step<<<ncta, 256, 0, c.stream>>>(n, bw, jb, L.d_band.p, L.d_bandL.p, L.d_dinv.p, L.d_jit.p, c.d_jitter.p);
    note_launch();
  }
  TM_CUDA_CHECK(cudaGetLastError());
  if (!try_band_inverse<8>(c, L) && !try_band_inverse<4>(c, L) && !try_band_inverse<2>(c, L) && !try_band_inverse<1>(c, L)) {
    k_band_inverse_warp<<<grid_for(n, 4), 128, 0, c.stream>>>(n, bw, L.d_bandL.p, L.d_inv.p);
    note_launch();
  }
  TM_CUDA_CHECK(cudaGetLastError());
}

}  // namespace tmg
