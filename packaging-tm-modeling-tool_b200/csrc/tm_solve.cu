// Solve-phase kernels: stencil apply, PCG vector work with deterministic reductions, and
// the multigrid V-cycle (MultigridPC._cycleOnce, src/core/10-solver.js:687-712).
//
// Differences from the reference, by design:
//  * the column Gauss-Seidel sweeps (columnSweep, 10-solver.js:512-555) visit the columns in
//    four colours (i mod 2, j mod 2) instead of lexicographically; columns of one colour do not
//    couple, so each colour is one parallel launch. Pre-smoothing runs colours 0..3, post-
//    smoothing 3..0, which keeps the V-cycle symmetric as the reference's forward/backward pair;
//  * the coarsest level is applied with the explicit inverse of its banded Cholesky factor;
//  * dot products are two-pass reductions in a fixed order (deterministic run to run).
#include <cuda_runtime.h>

#include <algorithm>

#include "tm_internal.h"
#include "tm_pdl.cuh"

namespace tmg {

namespace {

constexpr int RED_BLOCKS = 592;   // 4 x 148 SMs
constexpr int RED_THREADS = 256;

inline int grid_for(size_t n, int block) { return (int)((n + block - 1) / block); }

// ---- level-0 stencil apply: y = K x or y = b - K x over the positions p0 .. p1-1 -------------
// nn positions, slot-major arrays of row stride `stride`. Absent stencil slots hold exact zeros,
// so they read the node's own x (branch-free). NPT = 1:
// thread per position, the 27 neighbour ids fetched first. NPT = 2 or 4 (FP32 operator, row
// stride a multiple of 4): thread per aligned group of positions, every slot value of the group
// one vector load; the per-node arithmetic is the same for every NPT.
template <int NPT>
struct VecOf;
template <>
struct VecOf<2> { typedef float2 type; };
template <>
struct VecOf<4> { typedef float4 type; };
__device__ __forceinline__ float vcomp(const float2& v, int k) { return k == 0 ? v.x : v.y; }
__device__ __forceinline__ float vcomp(const float4& v, int k) { return k == 0 ? v.x : k == 1 ? v.y : k == 2 ? v.z : v.w; }

template <class T>
struct ApplyMinBlocks { static constexpr int value = 16; };
template <>
struct ApplyMinBlocks<float> { static constexpr int value = TM_APPLY32_MINB; };

template <class T, class V, int NPT>
__global__ void __launch_bounds__(128, ApplyMinBlocks<T>::value) k_apply0(int p0, int p1, int stride, int nn, const int* __restrict__ posNode,
                                                                         const int* __restrict__ nbr, const T* __restrict__ val,
                                                                         const V* __restrict__ x, V* __restrict__ y,
                                                                         const V* __restrict__ b) {
  if constexpr (NPT == 1) {
    const int ps = p0 + blockIdx.x * blockDim.x + threadIdx.x;
    if (ps >= p1) return;
    const int n = posNode[ps];
    T y0 = 0, y1 = 0, y2 = 0;
    int nb[NSLOT];
#pragma unroll
    for (int s = 0; s < NSLOT; s++) {
      const int j = nbr[(size_t)s * stride + ps];
      nb[s] = j < 0 ? n : j;
    }
#pragma unroll
    for (int s = 0; s < NSLOT; s++) {
      const size_t j = nb[s];
      const T x0 = (T)x[3 * j], x1 = (T)x[3 * j + 1], x2 = (T)x[3 * j + 2];
      const T* v = val + (size_t)s * 9 * stride + ps;
      y0 += v[0] * x0 + v[(size_t)stride] * x1 + v[2 * (size_t)stride] * x2;
      y1 += v[3 * (size_t)stride] * x0 + v[4 * (size_t)stride] * x1 + v[5 * (size_t)stride] * x2;
      y2 += v[6 * (size_t)stride] * x0 + v[7 * (size_t)stride] * x1 + v[8 * (size_t)stride] * x2;
    }
    if (b) {
      y[3 * n] = b[3 * n] - (V)y0; y[3 * n + 1] = b[3 * n + 1] - (V)y1; y[3 * n + 2] = b[3 * n + 2] - (V)y2;
    } else {
      y[3 * n] = (V)y0; y[3 * n + 1] = (V)y1; y[3 * n + 2] = (V)y2;
    }
  } else {
    static_assert((NPT == 2 || NPT == 4) && sizeof(T) == 4, "position groups are for the FP32 operator");
    typedef typename VecOf<NPT>::type VT;
    const int pa = (p0 & ~(NPT - 1)) + NPT * (blockIdx.x * blockDim.x + threadIdx.x);
    if (pa >= p1) return;
    // positions outside [p0, p1) are computed on valid memory (positions < nn, or the zero
    // padding of the operator rows) and not stored
    int n[NPT];
    T acc[NPT][3];
#pragma unroll
    for (int k = 0; k < NPT; k++) {
      n[k] = pa + k < nn ? posNode[pa + k] : 0;
      acc[k][0] = acc[k][1] = acc[k][2] = 0;
    }
    const size_t sv = (size_t)stride / NPT;
    TM_UNROLL(TM_APPLY32_UNROLL)
    for (int s = 0; s < NSLOT; s++) {
      T xv[NPT][3];
#pragma unroll
      for (int k = 0; k < NPT; k++) {
        const int jj = pa + k < nn ? nbr[(size_t)s * stride + pa + k] : -1;
        const size_t j = jj < 0 ? n[k] : jj;
        xv[k][0] = (T)x[3 * j]; xv[k][1] = (T)x[3 * j + 1]; xv[k][2] = (T)x[3 * j + 2];
      }
      const VT* v = reinterpret_cast<const VT*>(val + (size_t)s * 9 * stride + pa);
      VT vq[9];
#pragma unroll
      for (int q = 0; q < 9; q++) vq[q] = v[q * sv];
#pragma unroll
      for (int k = 0; k < NPT; k++)
#pragma unroll
        for (int r3 = 0; r3 < 3; r3++)
          acc[k][r3] += vcomp(vq[3 * r3], k) * xv[k][0] + vcomp(vq[3 * r3 + 1], k) * xv[k][1] + vcomp(vq[3 * r3 + 2], k) * xv[k][2];
    }
#pragma unroll
    for (int k = 0; k < NPT; k++) {
      if (pa + k < p0 || pa + k >= p1) continue;
      const size_t m = n[k];
      if (b) { y[3 * m] = b[3 * m] - (V)acc[k][0]; y[3 * m + 1] = b[3 * m + 1] - (V)acc[k][1]; y[3 * m + 2] = b[3 * m + 2] - (V)acc[k][2]; }
      else { y[3 * m] = (V)acc[k][0]; y[3 * m + 1] = (V)acc[k][1]; y[3 * m + 2] = (V)acc[k][2]; }
    }
  }
}

// threads of an apply over positions p0 .. p1-1
template <int NPT>
inline size_t apply_threads(int p0, int p1) {
  return (size_t)(p1 - (p0 & ~(NPT - 1)) + NPT - 1) / NPT;
}

// ---- deterministic reductions ----------------------------------------------------------------
template <class T>
__device__ double block_sum(double v) {
  __shared__ double sh[32];
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) sh[w] = v;
  __syncthreads();
  v = 0;
  if (threadIdx.x < 32) {
    v = threadIdx.x < (blockDim.x >> 5) ? sh[threadIdx.x] : 0;
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  }
  return v;
}

template <class T>
__global__ void k_dot_partial(size_t n, const T* __restrict__ a, const T* __restrict__ b, double* __restrict__ partial) {
  double s = 0;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) s += (double)a[i] * (double)b[i];
  s = block_sum<T>(s);
  if (threadIdx.x == 0) partial[blockIdx.x] = s;
}

__global__ void k_reduce_final(int np, const double* __restrict__ partial, double* __restrict__ out) {
  double s = 0;
  for (int i = threadIdx.x; i < np; i += blockDim.x) s += partial[i];
  s = block_sum<double>(s);
  if (threadIdx.x == 0) *out = s;
}

// all dots a_i . b_j of ma vectors a and mb vectors b (n entries each): each CTA walks chunks of
// MD_CHUNK entries (chunk c, c + grid, ...), stages the chunk of every vector in shared memory and
// adds the chunk's products to its threads' pairs (a thread starts its pair's row at its own
// offset, so the threads of a warp read different banks); partial[cta * np + p] then holds the
// CTA's sum of pair p = i * mb + j, and k_multi_dot_final adds the CTAs in order.
constexpr int MD_CHUNK = 128;
constexpr int MD_THREADS = 256;
constexpr int MD_MAXP = 2 * MD_THREADS;   // pairs per launch (two per thread)
constexpr int MD_MAXV = 200;              // vectors staged per launch (1 KB of shared memory each)
__global__ void __launch_bounds__(MD_THREADS) k_multi_dot_partial(size_t n, int ma, const double* const* __restrict__ A, int mb,
                                                                  const double* const* __restrict__ B, double* __restrict__ partial) {
  extern __shared__ double sh[];
  const int nv = ma + mb, np = ma * mb;
  double acc[2] = {0, 0};
  const size_t nchunks = (n + MD_CHUNK - 1) / MD_CHUNK;
  for (size_t ch = blockIdx.x; ch < nchunks; ch += gridDim.x) {
    const size_t r0 = ch * MD_CHUNK;
    const int len = (int)min((size_t)MD_CHUNK, n - r0);
    for (int e = threadIdx.x; e < nv * MD_CHUNK; e += MD_THREADS) {
      const int v = e / MD_CHUNK, t = e % MD_CHUNK;
      const double* src = v < ma ? A[v] : B[v - ma];
      sh[e] = t < len ? src[r0 + t] : 0.0;
    }
    __syncthreads();
#pragma unroll
    for (int u = 0; u < 2; u++) {
      const int p = threadIdx.x + u * MD_THREADS;
      if (p >= np) continue;
      const double* a = sh + (p / mb) * MD_CHUNK;
      const double* b = sh + (ma + p % mb) * MD_CHUNK;
      double s = 0;
      for (int t = 0; t < MD_CHUNK; t++) {
        const int q = (t + threadIdx.x) & (MD_CHUNK - 1);
        s += a[q] * b[q];
      }
      acc[u] += s;
    }
    __syncthreads();
  }
  for (int u = 0; u < 2; u++) {
    const int p = threadIdx.x + u * MD_THREADS;
    if (p < np) partial[(size_t)blockIdx.x * np + p] = acc[u];
  }
}
__global__ void k_multi_dot_final(int nblk, int np, const double* __restrict__ partial, double* __restrict__ out) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= np) return;
  double s = 0;
  for (int b = 0; b < nblk; b++) s += partial[(size_t)b * np + p];
  out[p] = s;
}

// x += alpha p ; r -= alpha q ; partial sums of r.r
template <class T>
__global__ void k_axpy2(size_t n, const double* __restrict__ alpha, const T* __restrict__ p, T* __restrict__ x, const T* __restrict__ q,
                        T* __restrict__ r, double* __restrict__ partial) {
  const T a = (T)*alpha;
  double s = 0;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    x[i] += a * p[i];
    const T ri = r[i] - a * q[i];
    r[i] = ri;
    s += (double)ri * (double)ri;
  }
  s = block_sum<T>(s);
  if (threadIdx.x == 0) partial[blockIdx.x] = s;
}

template <class T>
__global__ void k_xpby(size_t n, const T* __restrict__ z, const double* __restrict__ beta, T* __restrict__ p) {
  const T bt = (T)*beta;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) p[i] = z[i] + bt * p[i];
}

__global__ void k_div(const double* __restrict__ num, const double* __restrict__ den, double* __restrict__ out, double sign) {
  if (threadIdx.x == 0 && blockIdx.x == 0) *out = sign * (*num / *den);
}

template <class T>
__global__ void k_zero_list(int n, const int* __restrict__ idx, T* __restrict__ v) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) v[idx[i]] = 0;
}

template <class T>
__global__ void k_scale_vec(size_t n, const T* __restrict__ x, const double* __restrict__ s, T* __restrict__ y, int divide) {
  const size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (i < n) y[i] = divide ? (T)(x[i] / s[i]) : (T)(x[i] * s[i]);
}

// level-0 column smoother on packed column panels: one CTA per group of whole z-columns of one
// colour (at most cap nodes, contiguous in position order). Every thread computes the residual
// rows of one node (coalesced along each column's contiguous nodes), the column factors are
// staged in shared memory, one thread per column runs the block-tridiagonal forward/backward
// solve (solveColumn, 10-solver.js:71-104), and every node is then updated, x += dx.
template <class T>
struct PanelMinBlocks { static constexpr int value = TM_PANEL_MINB; };
template <>
struct PanelMinBlocks<double> { static constexpr int value = TM_PANEL_MINB_F64; };

template <class T>
__global__ void __launch_bounds__(TM_PANEL_THREADS, PanelMinBlocks<T>::value)
    k_sweep_panel(const int* __restrict__ grpStart, const int* __restrict__ colPos, const int* __restrict__ posNode, int nn,
                  const int* __restrict__ nbr, const T* __restrict__ val, const T* __restrict__ F, const T* __restrict__ b,
                  T* __restrict__ x, int cap, int zeroGuess) {
  extern __shared__ __align__(16) unsigned char smraw[];
  T* r = reinterpret_cast<T*>(smraw);            // 3*cap
  T* Fs = r + 3 * cap;                           // 18*cap
  int* off = reinterpret_cast<int*>(Fs + 18 * cap);   // node offsets of the group's columns (ncols + 1)
  const int g0 = grpStart[blockIdx.x], ncols = grpStart[blockIdx.x + 1] - g0;
  const int gp0 = colPos[g0];
  const int total = colPos[g0 + ncols] - gp0;
  for (int q = threadIdx.x; q <= ncols; q += blockDim.x) off[q] = colPos[g0 + q] - gp0;
  {
    const T* src = F + 18 * (size_t)gp0;
    for (int e = threadIdx.x; e < 18 * total; e += blockDim.x) Fs[e] = src[e];
  }
  for (int t = threadIdx.x; t < total; t += blockDim.x) {
    const int ps = gp0 + t;
    const int n = posNode[ps];
    T s0 = b[3 * (size_t)n], s1 = b[3 * (size_t)n + 1], s2 = b[3 * (size_t)n + 2];
    if (!zeroGuess) {
      // absent stencil slots hold exact zeros, so they read the node's own x (branch-free)
      TM_UNROLL(TM_PANEL_UNROLL)
      for (int s = 0; s < NSLOT; s++) {
        const int jj = nbr[(size_t)s * nn + ps];
        const size_t j = jj < 0 ? n : jj;
        const T x0 = x[3 * j], x1 = x[3 * j + 1], x2 = x[3 * j + 2];
        const T* v = val + (size_t)s * 9 * nn + ps;
        s0 -= v[0] * x0 + v[(size_t)nn] * x1 + v[2 * (size_t)nn] * x2;
        s1 -= v[3 * (size_t)nn] * x0 + v[4 * (size_t)nn] * x1 + v[5 * (size_t)nn] * x2;
        s2 -= v[6 * (size_t)nn] * x0 + v[7 * (size_t)nn] * x1 + v[8 * (size_t)nn] * x2;
      }
    }
    r[3 * t] = s0; r[3 * t + 1] = s1; r[3 * t + 2] = s2;
  }
  __syncthreads();
  for (int q = threadIdx.x; q < ncols; q += blockDim.x) {
    const int l0 = off[q], l1 = off[q + 1];
    for (int l = l0; l < l1; l++) {
      const T* f = Fs + 18 * l;
      T b0 = r[3 * l], b1 = r[3 * l + 1], b2 = r[3 * l + 2];
      if (l > l0) {
        const T p0 = r[3 * l - 3], p1 = r[3 * l - 2], p2 = r[3 * l - 1];
        b0 -= f[9] * p0 + f[10] * p1 + f[11] * p2;
        b1 -= f[12] * p0 + f[13] * p1 + f[14] * p2;
        b2 -= f[15] * p0 + f[16] * p1 + f[17] * p2;
      }
      const T y0 = b0 * f[1];
      const T y1 = (b1 - f[3] * y0) * f[2];
      const T y2 = (b2 - f[6] * y0 - f[7] * y1) * f[5];
      r[3 * l] = y0; r[3 * l + 1] = y1; r[3 * l + 2] = y2;
    }
    for (int l = l1 - 1; l >= l0; l--) {
      const T* f = Fs + 18 * l;
      T b0 = r[3 * l], b1 = r[3 * l + 1], b2 = r[3 * l + 2];
      if (l + 1 < l1) {
        const T* gg = Fs + 18 * (l + 1);
        const T q0 = r[3 * l + 3], q1 = r[3 * l + 4], q2 = r[3 * l + 5];
        b0 -= gg[9] * q0 + gg[12] * q1 + gg[15] * q2;
        b1 -= gg[10] * q0 + gg[13] * q1 + gg[16] * q2;
        b2 -= gg[11] * q0 + gg[14] * q1 + gg[17] * q2;
      }
      const T z2 = b2 * f[5];
      const T z1 = (b1 - f[7] * z2) * f[2];
      const T z0 = (b0 - f[3] * z1 - f[6] * z2) * f[1];
      r[3 * l] = z0; r[3 * l + 1] = z1; r[3 * l + 2] = z2;
    }
  }
  __syncthreads();
  for (int t = threadIdx.x; t < total; t += blockDim.x) {
    const size_t n = posNode[gp0 + t];
    x[3 * n] += r[3 * t]; x[3 * n + 1] += r[3 * t + 1]; x[3 * n + 2] += r[3 * t + 2];
  }
}

// restriction 0 -> 1: rc = P^T res, thread per (aggregate, component) over the aggregate's member
// nodes (ascending): the six threads of an aggregate share the members' residual loads and read
// adjacent weights, and each sums its component in the same order as a thread per aggregate would
template <class T>
__global__ void k_restrict0(int na, const int* __restrict__ aggPtr, const int* __restrict__ aggNodes, const T* __restrict__ W,
                            const T* __restrict__ res, T* __restrict__ rc, T* __restrict__ xc) {
  grid_dep_launch();
  const size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (t >= 6 * (size_t)na) return;
  const int I = (int)(t / 6), a = (int)(t % 6);
  xc[t] = 0;   // the level's iterate starts at zero
  T acc = 0;
  for (int q = aggPtr[I]; q < aggPtr[I + 1]; q++) {
    const int f = aggNodes[q];
    const T* w = W + 18 * (size_t)f;
    acc += w[a] * res[3 * f] + w[6 + a] * res[3 * f + 1] + w[12 + a] * res[3 * f + 2];
  }
  rc[t] = acc;
}

// prolongation 1 -> 0: x += P ec, thread per node
template <class T>
__global__ void k_prolong0(int nn, const int* __restrict__ nodeAgg, const T* __restrict__ W, const T* __restrict__ ec, T* __restrict__ x) {
  grid_dep_launch();
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= nn) return;
  const int a = nodeAgg[n];
  if (a < 0) return;   // a held node of a module stage: no prolongation
  const T* w = W + 18 * (size_t)n;
  const T* e = ec + 6 * (size_t)a;
#pragma unroll
  for (int p = 0; p < 3; p++) {
    T s = 0;
#pragma unroll
    for (int a = 0; a < 6; a++) s += w[p * 6 + a] * e[a];
    x[3 * (size_t)n + p] += s;
  }
}

// ---- shell levels (6x6 block CSR, a column's aggregates are a contiguous row range) -----------

// the 36 values of one 6x6 block with 16-byte loads (blocks start on 16-byte boundaries)
__device__ __forceinline__ void load_block36(const float* __restrict__ p, float (&v)[36]) {
  const float4* q = reinterpret_cast<const float4*>(p);
#pragma unroll
  for (int i = 0; i < 9; i++) {
    const float4 t = __ldg(q + i);
    v[4 * i] = t.x; v[4 * i + 1] = t.y; v[4 * i + 2] = t.z; v[4 * i + 3] = t.w;
  }
}
__device__ __forceinline__ void load_block36(const double* __restrict__ p, double (&v)[36]) {
  const double2* q = reinterpret_cast<const double2*>(p);
#pragma unroll
  for (int i = 0; i < 18; i++) {
    const double2 t = __ldg(q + i);
    v[2 * i] = t.x; v[2 * i + 1] = t.y;
  }
}

// rows of the column inverse a lane keeps in registers when the column block is small
constexpr int SH_PRE = 18;
// larger column inverses are staged in the warp's shared memory up to this size
constexpr size_t SH_AI_MAX = 12 * 1024;

// per-warp shared staging of the shell column kernels: the 6 partial sums of every block of the
// column's rows, the m residual rows (at least SH_PRE) and the local row starts
template <class T>
__host__ __device__ inline size_t shell_stage_bytes(int maxm, int maxBlk) {
  const int rlen = maxm > SH_PRE ? maxm : SH_PRE;
  const size_t b = sizeof(T) * (6 * (size_t)maxBlk + rlen) + sizeof(int) * ((size_t)maxm / 6 + 1);
  return (b + 15) / 16 * 16;
}
// whether a level's column inverses are staged in shared memory by the sweep, and the sweep's
// per-warp staging
template <class T>
__host__ __device__ inline bool shell_stage_ai(int maxm) {
  return maxm > SH_PRE && (size_t)maxm * maxm * sizeof(T) <= SH_AI_MAX;
}
template <class T>
__host__ __device__ inline size_t shell_sweep_bytes(int maxm, int maxBlk, bool stageAi) {
  return shell_stage_bytes<T>(maxm, maxBlk) + (stageAi ? ((size_t)maxm * maxm * sizeof(T) + 15) / 16 * 16 : 0);
}

// residual rows r = b - K x of the column whose aggregates are n0 .. n0+na-1 (blocks k0 ..
// k0+nblk-1), by one warp: the lanes take the column's blocks (all rows together), each lane's 6
// products of a block land in shared memory, and lane e then subtracts its row's block sums in
// block order, as the serial row loop of columnSweep (10-solver.js:535-553) does. A lane's blocks
// are taken SH_BPL at a time: first all their column indices, then all their neighbour values,
// then the block values and the products, so that each of these steps is one round of loads
// rather than one per block.
//
// Two parts. shell_column_static reads what the V-cycle never writes: the local row starts, the
// first round of block column indices (cj0) and an L2 prefetch of the first round's blocks; it
// runs before the grid-dependency wait. shell_column_residual runs after it (b and x).
constexpr int SH_BPL = 4;
template <class T>
__device__ __forceinline__ void shell_column_static(int lane, int n0, int na, int k0, int nblk, const int* __restrict__ rowPtr,
                                                    const int* __restrict__ col, const T* __restrict__ val, bool zeroGuess,
                                                    int* rp, int (&cj0)[SH_BPL]) {
#pragma unroll
  for (int u = 0; u < SH_BPL; u++) cj0[u] = -1;
  if (zeroGuess) return;
  for (int q = lane; q <= na; q += 32) rp[q] = rowPtr[n0 + q] - k0;
#pragma unroll
  for (int u = 0; u < SH_BPL; u++) {
    const int e = lane + 32 * u;
    if (e < nblk) {
      cj0[u] = col[k0 + e];
      const char* blk = reinterpret_cast<const char*>(val + 36 * (size_t)(k0 + e));
      asm volatile("prefetch.global.L2 [%0];\n" ::"l"(blk));
      asm volatile("prefetch.global.L2 [%0];\n" ::"l"(blk + 36 * sizeof(T) - 1));
    }
  }
}
template <class T>
__device__ __forceinline__ void shell_column_residual(int lane, int n0, int na, int k0, int nblk, const int* __restrict__ col,
                                                      const T* __restrict__ val, const T* __restrict__ b, const T* __restrict__ x,
                                                      bool zeroGuess, const int (&cj0)[SH_BPL], T* part, T* r, const int* rp) {
  const int m = 6 * na;
  // the column's b is loaded with the block rows, not after them
  const T* bc = b + 6 * (size_t)n0;
  const T bo0 = lane < m ? __ldcg(bc + lane) : (T)0, bo1 = lane + 32 < m ? __ldcg(bc + lane + 32) : (T)0;
  auto bval = [&](int e) { return e == lane ? bo0 : e == lane + 32 ? bo1 : __ldcg(bc + e); };
  if (zeroGuess) {
    for (int e = lane; e < m; e += 32) r[e] = bval(e);
    __syncwarp();
    return;
  }
  for (int e0 = 0; e0 < nblk; e0 += 32 * SH_BPL) {
    int cj[SH_BPL];
#pragma unroll
    for (int u = 0; u < SH_BPL; u++) {
      const int e = e0 + lane + 32 * u;
      cj[u] = e0 == 0 ? cj0[u] : e < nblk ? col[k0 + e] : -1;
    }
    T xv[SH_BPL][6];
#pragma unroll
    for (int u = 0; u < SH_BPL; u++) {
      const T* xj = x + 6 * (size_t)(cj[u] < 0 ? 0 : cj[u]);
#pragma unroll
      for (int q = 0; q < 6; q++) xv[u][q] = cj[u] >= 0 ? __ldcg(xj + q) : (T)0;
    }
#pragma unroll
    for (int u = 0; u < SH_BPL; u++) {
      const int e = e0 + lane + 32 * u;
      if (e >= nblk) break;
      T v[36];
      load_block36(val + 36 * (size_t)(k0 + e), v);
#pragma unroll
      for (int p = 0; p < 6; p++)
        part[6 * e + p] = v[6 * p] * xv[u][0] + v[6 * p + 1] * xv[u][1] + v[6 * p + 2] * xv[u][2] + v[6 * p + 3] * xv[u][3] +
                          v[6 * p + 4] * xv[u][4] + v[6 * p + 5] * xv[u][5];
    }
  }
  __syncwarp();
  for (int e = lane; e < m; e += 32) {
    const int a = e / 6, p = e % 6;
    T s = bval(e);
    for (int k = rp[a]; k < rp[a + 1]; k++) s -= part[6 * k + p];
    r[e] = s;
  }
  __syncwarp();
}

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(gmem) : "memory");
}

// one column of a shell-level sweep by one warp: r = b - K x over the column's rows, then
// x_col += A_cc^-1 r with the explicit inverse Ai (entry (e, k) at k*m + e). The inverse reaches the
// lanes before the residual is done: rows of at most SH_PRE entries in registers, larger blocks
// copied asynchronously into the warp's shared memory (aiSm, when the level's blocks fit there) and
// otherwise read from global memory after it. The inverse, the row starts and the first block
// columns are read before the grid-dependency wait (no kernel of the V-cycle writes them); b and x
// after it. Every lane fetches its entries of the column's own x right after the wait: no other
// warp writes this column's x during the launch (a colour's columns do not couple), and this warp
// writes it only at the end.
template <class T>
__device__ __forceinline__ void shell_sweep_column(int lane, int4 mt, const T* __restrict__ Ai, const int* __restrict__ rowPtr,
                                                   const int* __restrict__ col, const T* __restrict__ val, const T* __restrict__ b,
                                                   T* __restrict__ x, bool zeroGuess, T* part, T* r, int* rp, T* aiSm) {
  const int n0 = mt.x, na = mt.y - mt.x, m = 6 * na;
  T a[SH_PRE];
  const bool pre = m <= SH_PRE;
#pragma unroll
  for (int k = 0; k < SH_PRE; k++) a[k] = (pre && lane < m && k < m) ? Ai[(size_t)k * m + lane] : (T)0;
  const bool staged = !pre && aiSm != nullptr;
  if (staged) {
    // m*m values, a multiple of 36: 16-byte pieces (the block starts on a 16-byte boundary)
    const int pieces = m * m * (int)sizeof(T) / 16;
    for (int q = lane; q < pieces; q += 32) cp_async16(reinterpret_cast<unsigned char*>(aiSm) + 16 * q, reinterpret_cast<const unsigned char*>(Ai) + 16 * q);
    asm volatile("cp.async.commit_group;\n" ::: "memory");
  }
  int cj0[SH_BPL];
  shell_column_static(lane, n0, na, mt.z, mt.w - mt.z, rowPtr, col, val, zeroGuess, rp, cj0);
  grid_dep_wait();
  T* xc = x + 6 * (size_t)n0;
  const T xo0 = lane < m ? __ldcg(xc + lane) : (T)0, xo1 = lane + 32 < m ? __ldcg(xc + lane + 32) : (T)0;
  shell_column_residual(lane, n0, na, mt.z, mt.w - mt.z, col, val, b, x, zeroGuess, cj0, part, r, rp);
  if (pre) {
    if (lane < m) {
      T acc = 0;
#pragma unroll
      for (int k = 0; k < SH_PRE; k++)
        if (k < m) acc += a[k] * r[k];
      xc[lane] = xo0 + acc;
    }
    return;
  }
  const T* A = Ai;
  if (staged) {
    asm volatile("cp.async.wait_all;\n" ::: "memory");
    __syncwarp();
    A = aiSm;
  }
  for (int e = lane; e < m; e += 32) {
    T acc = 0;
#pragma unroll 6
    for (int k = 0; k < m; k++) acc += A[(size_t)k * m + e] * r[k];
    xc[e] = (e == lane ? xo0 : e == lane + 32 ? xo1 : __ldcg(xc + e)) + acc;
  }
}

// shell-level residual res = b - K x over all columns, warp per column (meta: first and
// one-past-last aggregate and block of every column); launched with a programmatic dependency on
// the level's last sweep
template <class T>
__global__ void __launch_bounds__(256) k_apply_shell(int ncol, const int4* __restrict__ meta, const int* __restrict__ rowPtr,
                                                     const int* __restrict__ col, const T* __restrict__ val, const T* __restrict__ x,
                                                     const T* __restrict__ b, T* __restrict__ y, int maxm, int maxBlk) {
  extern __shared__ __align__(16) unsigned char smraw[];
  grid_dep_launch();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int c = blockIdx.x * (blockDim.x >> 5) + warp;
  if (c >= ncol) return;
  unsigned char* base = smraw + (size_t)warp * shell_stage_bytes<T>(maxm, maxBlk);
  T* part = reinterpret_cast<T*>(base);
  T* r = part + 6 * (size_t)maxBlk;
  int* rp = reinterpret_cast<int*>(r + (maxm > SH_PRE ? maxm : SH_PRE));
  const int4 mt = meta[c];
  const int n0 = mt.x, na = mt.y - mt.x;
  int cj0[SH_BPL];
  shell_column_static(lane, n0, na, mt.z, mt.w - mt.z, rowPtr, col, val, false, rp, cj0);
  grid_dep_wait();
  shell_column_residual(lane, n0, na, mt.z, mt.w - mt.z, col, val, b, x, false, cj0, part, r, rp);
  for (int e = lane; e < 6 * na; e += 32) y[6 * (size_t)n0 + e] = r[e];
}

// shell-level column sweep, warp per column of one colour (columnSweep shell branch,
// 10-solver.js:535-553): r = b - K x over the column's rows, then x_col += A_cc^-1 r with the
// explicit inverse of the column block. The colour's column list carries each column's aggregate
// and block ranges and the offset of its inverse (one load). Launched with a programmatic
// dependency on the previous kernel, so its reads of the column structure overlap that kernel.
template <class T>
__global__ void __launch_bounds__(256) k_sweep_shell(int ncolc, const int4* __restrict__ meta, const long long* __restrict__ cfOff,
                                                     const int* __restrict__ rowPtr, const int* __restrict__ col,
                                                     const T* __restrict__ val, const T* __restrict__ cf, const T* __restrict__ b,
                                                     T* __restrict__ x, int maxm, int maxBlk, int zeroGuess, int stageAi) {
  extern __shared__ __align__(16) unsigned char smraw[];
  grid_dep_launch();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int gw = blockIdx.x * (blockDim.x >> 5) + warp;
  if (gw >= ncolc) return;
  unsigned char* base = smraw + (size_t)warp * shell_sweep_bytes<T>(maxm, maxBlk, stageAi != 0);
  T* part = reinterpret_cast<T*>(base);
  T* r = part + 6 * (size_t)maxBlk;
  int* rp = reinterpret_cast<int*>(r + (maxm > SH_PRE ? maxm : SH_PRE));
  T* aiSm = stageAi ? reinterpret_cast<T*>(base + shell_stage_bytes<T>(maxm, maxBlk)) : nullptr;
  shell_sweep_column<T>(lane, meta[gw], cf + cfOff[gw], rowPtr, col, val, b, x, zeroGuess != 0, part, r, rp, aiSm);
}

// shell restriction: rc = P^T res (children lists, transposeProl order)
template <class T>
__global__ void k_restrict_shell(int nnc, const int* __restrict__ chPtr, const int* __restrict__ chIdx, const int* __restrict__ chW,
                                 const T* __restrict__ W, const T* __restrict__ res, T* __restrict__ rc, T* __restrict__ xc) {
  grid_dep_launch();
  const size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (t >= 6 * (size_t)nnc) return;
  xc[t] = 0;   // the coarse level's iterate starts at zero
  const int I = (int)(t / 6), a = (int)(t % 6);
  T acc = 0;
  for (int q = chPtr[I]; q < chPtr[I + 1]; q++) {
    const int f = chIdx[q];
    const T* w = W + 36 * (size_t)chW[q];
    const T* r = res + 6 * (size_t)f;
    acc += w[a] * r[0] + w[6 + a] * r[1] + w[12 + a] * r[2] + w[18 + a] * r[3] + w[24 + a] * r[4] + w[30 + a] * r[5];
  }
  rc[t] = acc;
}

// shell prolongation: x += P ec
template <class T>
__global__ void k_prolong_shell(int nnf, const int* __restrict__ prolPtr, const int* __restrict__ prolIdx, const T* __restrict__ W,
                                const T* __restrict__ ec, T* __restrict__ x) {
  grid_dep_launch();
  const size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (t >= 6 * (size_t)nnf) return;
  const int f = (int)(t / 6), p = (int)(t % 6);
  T v = x[t];
  for (int q = prolPtr[f]; q < prolPtr[f + 1]; q++) {
    const T* w = W + 36 * (size_t)q + 6 * p;
    const T* e = ec + 6 * (size_t)prolIdx[q];
    v += w[0] * e[0] + w[1] * e[1] + w[2] * e[2] + w[3] * e[3] + w[4] * e[4] + w[5] * e[5];
  }
  x[t] = v;
}

// coarsest: x = A^-1 b with the explicit inverse, warp per row
template <class T, class M>
__global__ void k_dense_apply(int n, const M* __restrict__ inv, const T* __restrict__ b, T* __restrict__ x) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int i = blockIdx.x * (blockDim.x >> 5) + warp;
  if (i >= n) return;
  double s = 0;
  for (int k = lane; k < n; k += 32) s += (double)inv[(size_t)i * n + k] * (double)b[k];
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  if (lane == 0) x[i] = (T)s;
}

__global__ void k_axpy_scalar(size_t n, double alpha, const double* __restrict__ x, double* __restrict__ y) {
  const size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (i < n) y[i] += alpha * x[i];
}

__global__ void k_div_scalar(size_t n, double* __restrict__ v, double d) {
  const size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (i < n) v[i] /= d;
}

template <class A, class B>
__global__ void k_convert(size_t n, const A* __restrict__ a, B* __restrict__ b) {
  const size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (i < n) b[i] = (B)a[i];
}

__global__ void k_add_f2d(size_t n, const float* __restrict__ d, double* __restrict__ x) {
  const size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (i < n) x[i] += (double)d[i];
}

// buffers of one precision of the V-cycle
template <class T>
struct Bufs;
template <>
struct Bufs<double> {
  static const double* val0(Context& c) { return c.d_val.p; }
  static const double* F(Context& c) { return c.d_F.p; }
  static const double* W01(Context& c) { return c.d_W01.p; }
  static double* res0(Context& c) { return c.d_res0.p; }
  static const double* val(ShellLevel& L) { return L.d_val.p; }
  static const double* cf(ShellLevel& L) { return L.d_cfInv.p; }
  static const double* prolW(ShellLevel& L) { return L.d_prolW.p; }
  static double* b(ShellLevel& L) { return L.d_b.p; }
  static double* x(ShellLevel& L) { return L.d_x.p; }
  static double* res(ShellLevel& L) { return L.d_res.p; }
};
template <>
struct Bufs<float> {
  static const float* val0(Context& c) { return c.d_val32.p; }
  static const float* F(Context& c) { return c.d_F32.p; }
  static const float* W01(Context& c) { return c.d_W01_32.p; }
  static float* res0(Context& c) { return c.d_res0_32.p; }
  static const float* val(ShellLevel& L) { return L.d_val32.p; }
  static const float* cf(ShellLevel& L) { return L.d_cfInv32.p; }
  static const float* prolW(ShellLevel& L) { return L.d_prolW32.p; }
  static float* b(ShellLevel& L) { return L.d_b32.p; }
  static float* x(ShellLevel& L) { return L.d_x32.p; }
  static float* res(ShellLevel& L) { return L.d_res32.p; }
};

// y = K x (or b - K x) over the positions p0 .. p1-1: FP32 operators in position groups, FP64
// operators one position per thread
template <class T, class V>
void apply0_range(Context& c, const T* val, int p0, int p1, const V* x, V* y, const V* b) {
  if (p1 <= p0) return;
  if constexpr (sizeof(T) == 4)
    k_apply0<T, V, TM_APPLY32_NPT><<<grid_for(apply_threads<TM_APPLY32_NPT>(p0, p1), 128), 128, 0, c.stream>>>(p0, p1, c.nnp, c.nn,
        c.d_posNode.p, c.d_nbr.p, val, x, y, b);
  else
    k_apply0<T, V, 1><<<grid_for(apply_threads<1>(p0, p1), 128), 128, 0, c.stream>>>(p0, p1, c.nnp, c.nn, c.d_posNode.p, c.d_nbr.p, val, x,
        y, b);
  note_launch();
}

// MultigridPC._cycleOnce (10-solver.js:687-712) with zero initial guess on every level
template <class T>
void vcycle(Context& c, const T* r, T* z) {
  typedef Bufs<T> B;
  cudaStream_t st = c.stream;
  const int nn = c.nn;
  const size_t smem0 = (size_t)21 * c.panelCap * sizeof(T) + (size_t)(c.panelMaxCols + 1) * sizeof(int);
  // the iterate starts at zero (the TMA sweep clears it itself on the first sweep)
  if (sizeof(T) == 8 || !c.tsReady || c.mf) TM_CUDA_CHECK(cudaMemsetAsync(z, 0, 3 * (size_t)nn * sizeof(T), st));
  if (smem0 > 48 * 1024) TM_CUDA_CHECK(cudaFuncSetAttribute(k_sweep_panel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem0));
  auto sweep0 = [&](int col, int zero) {
    if (!c.grpCount[col]) return;
    TimedLaunch tl(c, K_SWEEP_SOLID);
    if (c.mf) {   // level 0 from the cell-class table
      if constexpr (sizeof(T) == 4) launch_mf_sweep32(c, col, zero, (const float*)r, (float*)z);
      else launch_mf_sweep64(c, col, zero, (const double*)r, (double*)z);
      return;
    }
    if constexpr (sizeof(T) == 4)
      if (launch_sweep_tma(c, col, zero, r, z)) return;
    k_sweep_panel<T><<<c.grpCount[col], TM_PANEL_THREADS, smem0, st>>>(c.d_grpStart[col].p, c.d_colPos[col].p, c.d_posNode.p, c.nnp,
        c.d_nbr.p, B::val0(c), B::F(c), r, z, c.panelCap, zero);
    note_launch();
  };
  // warps per block of the shell kernels: 4, or the autotuned shapes of the FP32 cycle
  auto wpbS = [&](const ShellLevel& L) { return sizeof(T) == 4 ? L.wpbSweep : 4; };
  auto wpbA = [&](const ShellLevel& L) { return sizeof(T) == 4 ? L.wpbApply : 4; };
  size_t smemS = 0;
  for (auto& Lp : c.shells)
    smemS = std::max(smemS, (size_t)std::max(wpbS(*Lp), wpbA(*Lp)) *
                                shell_sweep_bytes<T>(Lp->maxm, Lp->maxColBlocks, shell_stage_ai<T>(Lp->maxm)));
  if (smemS > 48 * 1024) {
    TM_CUDA_CHECK(cudaFuncSetAttribute(k_sweep_shell<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smemS));
    TM_CUDA_CHECK(cudaFuncSetAttribute(k_apply_shell<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smemS));
  }
  auto sweepS = [&](ShellLevel& L, int col, int zero) {
    const bool sai = shell_stage_ai<T>(L.maxm);
    const size_t per = shell_sweep_bytes<T>(L.maxm, L.maxColBlocks, sai);
    const int wpb = wpbS(L);
    TimedLaunch tl(c, K_SWEEP_SHELL);
    launch_pdl(k_sweep_shell<T>, grid_for(L.colorCount[col], wpb), 32 * wpb, wpb * per, st, L.colorCount[col],
               (const int4*)L.d_colorMeta[col].p, (const long long*)L.d_colorCf[col].p, (const int*)L.d_rowPtr.p, (const int*)L.d_col.p,
               (const T*)B::val(L), (const T*)B::cf(L), (const T*)B::b(L), B::x(L), L.maxm, L.maxColBlocks, zero, sai ? 1 : 0);
    note_launch();
  };
  // ---- level 0 pre-smoothing: 2 sweeps in colours 0..3
  bool first = true;
  for (int sw = 0; sw < 2; sw++)
    for (int col = 0; col < 4; col++) {
      if (!c.colorCount[col]) continue;
      sweep0(col, first ? 1 : 0);
      first = false;
    }
  {
    TimedLaunch tl(c, K_APPLY0);
    if (c.mf) {
      if constexpr (sizeof(T) == 4) launch_mf_apply32(c, (const float*)z, (float*)B::res0(c), (const float*)r);
      else launch_mf_apply(c, (const double*)z, (double*)B::res0(c), (const double*)r);
    } else {
      apply0_range<T, T>(c, B::val0(c), 0, nn, z, B::res0(c), r);
    }
  }
  ShellLevel& L1 = *c.shells[0];
  k_restrict0<T><<<grid_for(6 * (size_t)L1.nn, 192), 192, 0, st>>>(L1.nn, c.d_aggPtr.p, c.d_aggNodes.p, B::W01(c), B::res0(c),
                                                                     B::b(L1), B::x(L1));
  note_launch();
  const size_t nl = c.shells.size();
  for (size_t l = 0; l < nl; l++) {
    ShellLevel& L = *c.shells[l];
    if (L.coarsest) {
      // coarsest-grid direct solve in FP64 whatever the precision of the cycle
      k_dense_apply<T, double><<<grid_for(L.denseN, 4), 128, 0, st>>>(L.denseN, L.d_inv.p, B::b(L), B::x(L));
      note_launch();
      break;
    }
    bool firstS = true;   // the level's iterate was cleared by the restriction that made its b
    for (int sw = 0; sw < 2; sw++)
      for (int col = 0; col < 4; col++) {
        if (!L.colorCount[col]) continue;
        sweepS(L, col, firstS ? 1 : 0);
        firstS = false;
      }
    {
      TimedLaunch tl(c, K_APPLY_SHELL);
      const int ncol = L.nx * L.ny;
      const int wpb = wpbA(L);
      launch_pdl(k_apply_shell<T>, grid_for(ncol, wpb), 32 * wpb, wpb * shell_stage_bytes<T>(L.maxm, L.maxColBlocks), st, ncol,
                 (const int4*)L.d_colMeta.p, (const int*)L.d_rowPtr.p, (const int*)L.d_col.p, (const T*)B::val(L), (const T*)B::x(L),
                 (const T*)B::b(L), B::res(L), L.maxm, L.maxColBlocks);
      note_launch();
    }
    ShellLevel& C = *c.shells[l + 1];
    k_restrict_shell<T><<<grid_for(6 * (size_t)C.nn, 128), 128, 0, st>>>(C.nn, L.d_chPtr.p, L.d_chIdx.p, L.d_chW.p, B::prolW(L), B::res(L),
        B::b(C), B::x(C));
    note_launch();
  }
  for (int l = (int)nl - 2; l >= 0; l--) {
    ShellLevel& L = *c.shells[l];
    ShellLevel& C = *c.shells[l + 1];
    k_prolong_shell<T><<<grid_for(6 * (size_t)L.nn, 128), 128, 0, st>>>(L.nn, L.d_prolPtr.p, L.d_prolIdx.p, B::prolW(L), B::x(C), B::x(L));
    note_launch();
    for (int sw = 0; sw < 2; sw++)
      for (int col = 3; col >= 0; col--)
        if (L.colorCount[col]) sweepS(L, col, 0);
  }
  // ---- level 0: prolongation and post-smoothing, colours 3..0
  k_prolong0<T><<<grid_for(nn, 128), 128, 0, st>>>(nn, c.d_nodeAgg.p, B::W01(c), B::x(L1), z);
  note_launch();
  for (int sw = 0; sw < 2; sw++)
    for (int col = 3; col >= 0; col--)
      if (c.colorCount[col]) sweep0(col, 0);
  TM_CUDA_CHECK(cudaGetLastError());
}

}  // namespace

// ---- launch accounting and event timers ----------------------------------------------------------
static long long g_launches = 0;
void note_launch(int count) { __atomic_fetch_add(&g_launches, (long long)count, __ATOMIC_RELAXED); }
long long launch_count() { return __atomic_load_n(&g_launches, __ATOMIC_RELAXED); }

TimedLaunch::TimedLaunch(Context& ctx, int kid) : c(ctx), on(ctx.timerKernel == kid) {
  if (!on) return;
  TM_CUDA_CHECK(cudaEventCreate(&a));
  TM_CUDA_CHECK(cudaEventCreate(&b));
  TM_CUDA_CHECK(cudaEventRecord(a, c.stream));
}
TimedLaunch::~TimedLaunch() {
  if (!on) return;
  cudaEventRecord(b, c.stream);
  c.timerEvents.emplace_back(a, b);
}

void launch_apply0(Context& c, const double* x, double* y, const double* b) {
  TimedLaunch tl(c, K_APPLY0);
  if (c.mf) { launch_mf_apply(c, x, y, b); return; }
  apply0_range<double, double>(c, c.d_val.p, 0, c.nn, x, y, b);
  TM_CUDA_CHECK(cudaGetLastError());
}

void launch_apply0_f32(Context& c, const double* x, double* y, const double* b) {
  apply0_range<float, double>(c, c.d_val32.p, 0, c.nn, x, y, b);
  TM_CUDA_CHECK(cudaGetLastError());
}

void launch_apply0_32(Context& c, const float* x, float* y, const float* b) {
  TimedLaunch tl(c, K_APPLY0);
  if (c.mf) { launch_mf_apply32(c, x, y, b); return; }
  apply0_range<float, float>(c, c.d_val32.p, 0, c.nn, x, y, b);
  TM_CUDA_CHECK(cudaGetLastError());
}

void launch_dot(Context& c, const double* a, const double* b, size_t n, double* out_dev) {
  k_dot_partial<double><<<RED_BLOCKS, RED_THREADS, 0, c.stream>>>(n, a, b, c.d_partial.p);
  k_reduce_final<<<1, 1024, 0, c.stream>>>(RED_BLOCKS, c.d_partial.p, out_dev);
  note_launch(2);
  TM_CUDA_CHECK(cudaGetLastError());
}

void multi_dot_host(Context& c, const std::vector<const double*>& a, const std::vector<const double*>& b, size_t n, double* out) {
  const int ma = (int)a.size(), mb = (int)b.size(), np = ma * mb;
  if (!np) return;
  // a launch holds at most MD_MAXP pairs and MD_MAXV staged vectors (MD_MAXV KB of shared memory)
  if (mb > MD_MAXV / 2) fail(TM_BAD_INPUT, "too many vectors for one batched dot launch");
  const int rows = std::min(MD_MAXP / mb, MD_MAXV - mb);
  if (ma > rows) {   // rows of a in groups that fit one launch
    for (int i0 = 0; i0 < ma; i0 += rows) {
      const std::vector<const double*> part(a.begin() + i0, a.begin() + std::min(ma, i0 + rows));
      multi_dot_host(c, part, b, n, out + (size_t)i0 * mb);
    }
    return;
  }
  std::vector<const double*> ptr(a);
  ptr.insert(ptr.end(), b.begin(), b.end());
  if (c.d_mdPtr.n < (size_t)MD_MAXV) c.d_mdPtr.alloc(MD_MAXV);
  TM_CUDA_CHECK(cudaMemcpyAsync(c.d_mdPtr.p, ptr.data(), ptr.size() * sizeof(uintptr_t), cudaMemcpyHostToDevice, c.stream));
  const int blocks = RED_BLOCKS / 2;
  c.d_mdPart.alloc((size_t)blocks * MD_MAXP + MD_MAXP);
  const double* const* P = reinterpret_cast<const double* const*>(c.d_mdPtr.p);
  const size_t smem = (size_t)(ma + mb) * MD_CHUNK * sizeof(double);
  if (smem > 48 * 1024) TM_CUDA_CHECK(cudaFuncSetAttribute(k_multi_dot_partial, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  double* fin = c.d_mdPart.p + (size_t)blocks * MD_MAXP;
  k_multi_dot_partial<<<blocks, MD_THREADS, smem, c.stream>>>(n, ma, P, mb, P + ma, c.d_mdPart.p);
  k_multi_dot_final<<<grid_for(np, 128), 128, 0, c.stream>>>(blocks, np, c.d_mdPart.p, fin);
  note_launch(2);
  TM_CUDA_CHECK(cudaGetLastError());
  TM_CUDA_CHECK(cudaMemcpyAsync(out, fin, np * sizeof(double), cudaMemcpyDeviceToHost, c.stream));
  TM_CUDA_CHECK(cudaStreamSynchronize(c.stream));
}

void launch_dot32(Context& c, const float* a, const float* b, size_t n, double* out_dev) {
  k_dot_partial<float><<<RED_BLOCKS, RED_THREADS, 0, c.stream>>>(n, a, b, c.d_partial.p);
  k_reduce_final<<<1, 1024, 0, c.stream>>>(RED_BLOCKS, c.d_partial.p, out_dev);
  note_launch(2);
  TM_CUDA_CHECK(cudaGetLastError());
}

void launch_finalize(Context& c, double* out_dev) {
  k_reduce_final<<<1, 1024, 0, c.stream>>>(RED_BLOCKS, c.d_partial.p, out_dev);
  note_launch();
  TM_CUDA_CHECK(cudaGetLastError());
}

void launch_axpy(Context& c, double alpha, const double* x, double* y, size_t n) {
  k_axpy_scalar<<<grid_for(n, 256), 256, 0, c.stream>>>(n, alpha, x, y);
  note_launch();
  TM_CUDA_CHECK(cudaGetLastError());
}

void launch_div_scalar(Context& c, double* v, double d, size_t n) {
  k_div_scalar<<<grid_for(n, 256), 256, 0, c.stream>>>(n, v, d);
  note_launch();
  TM_CUDA_CHECK(cudaGetLastError());
}

void launch_axpy2(Context& c, const double* alpha_dev, const double* p, double* x, const double* q, double* r, size_t n) {
  k_axpy2<double><<<RED_BLOCKS, RED_THREADS, 0, c.stream>>>(n, alpha_dev, p, x, q, r, c.d_partial.p);
  note_launch();
  TM_CUDA_CHECK(cudaGetLastError());
}

void launch_axpy2_32(Context& c, const double* alpha_dev, const float* p, float* x, const float* q, float* r, size_t n) {
  k_axpy2<float><<<RED_BLOCKS, RED_THREADS, 0, c.stream>>>(n, alpha_dev, p, x, q, r, c.d_partial.p);
  note_launch();
  TM_CUDA_CHECK(cudaGetLastError());
}

void launch_xpby(Context& c, const double* z, const double* beta_dev, double* p, size_t n) {
  k_xpby<double><<<RED_BLOCKS, RED_THREADS, 0, c.stream>>>(n, z, beta_dev, p);
  note_launch();
  TM_CUDA_CHECK(cudaGetLastError());
}

void launch_xpby32(Context& c, const float* z, const double* beta_dev, float* p, size_t n) {
  k_xpby<float><<<RED_BLOCKS, RED_THREADS, 0, c.stream>>>(n, z, beta_dev, p);
  note_launch();
  TM_CUDA_CHECK(cudaGetLastError());
}

void launch_div(Context& c, const double* num, const double* den, double* out, double sign) {
  k_div<<<1, 32, 0, c.stream>>>(num, den, out, sign);
  note_launch();
  TM_CUDA_CHECK(cudaGetLastError());
}

void launch_zero_constrained(Context& c, double* v) {
  if (c.constr.empty()) return;
  k_zero_list<double><<<grid_for(c.constr.size(), 128), 128, 0, c.stream>>>((int)c.constr.size(), c.d_constr.p, v);
  note_launch();
  TM_CUDA_CHECK(cudaGetLastError());
}

void launch_zero_constrained32(Context& c, float* v) {
  if (c.constr.empty()) return;
  k_zero_list<float><<<grid_for(c.constr.size(), 128), 128, 0, c.stream>>>((int)c.constr.size(), c.d_constr.p, v);
  note_launch();
  TM_CUDA_CHECK(cudaGetLastError());
}

void launch_scale_vec(Context& c, const double* x, const double* s, double* y, bool divide, size_t n) {
  k_scale_vec<double><<<grid_for(n, 256), 256, 0, c.stream>>>(n, x, s, y, divide ? 1 : 0);
  note_launch();
  TM_CUDA_CHECK(cudaGetLastError());
}

void launch_d2f(Context& c, const double* a, float* b, size_t n) {
  k_convert<double, float><<<grid_for(n, 256), 256, 0, c.stream>>>(n, a, b);
  note_launch();
  TM_CUDA_CHECK(cudaGetLastError());
}

void launch_f2d(Context& c, const float* a, double* b, size_t n) {
  k_convert<float, double><<<grid_for(n, 256), 256, 0, c.stream>>>(n, a, b);
  note_launch();
  TM_CUDA_CHECK(cudaGetLastError());
}

void launch_add_f2d(Context& c, const float* d, double* x, size_t n) {
  k_add_f2d<<<grid_for(n, 256), 256, 0, c.stream>>>(n, d, x);
  note_launch();
  TM_CUDA_CHECK(cudaGetLastError());
}

// the V-cycle replayed from a CUDA graph (about 130 launches of mostly small kernels per cycle);
// launched directly while a kernel class is being timed (the timer's events are per launch)
template <class T>
void vcycle_graph(Context& c, const T* r, T* z) {
  if (c.timerKernel >= 0) {
    vcycle<T>(c, r, z);
    return;
  }
  const int idx = sizeof(T) == 4 ? 1 : 0;
  size_t key = 1469598103934665603ull;
  for (size_t v : {(size_t)r, (size_t)z, (size_t)c.structEpoch, (size_t)c.shapeEpoch, (size_t)Bufs<T>::val0(c), (size_t)c.stream,
                   (size_t)c.mf, (size_t)c.d_ccK32.p, (size_t)c.d_gs32.p, (size_t)c.d_gs.p})
    key = (key ^ v) * 1099511628211ull;
  if (!c.vcGraph[idx] || c.vcKey[idx] != key) {
    if (c.vcGraph[idx]) {
      TM_CUDA_CHECK(cudaGraphExecDestroy(c.vcGraph[idx]));
      c.vcGraph[idx] = nullptr;
    }
    if (!c.capStream) TM_CUDA_CHECK(cudaStreamCreateWithFlags(&c.capStream, cudaStreamNonBlocking));
    // the caller's stream may be the legacy default stream, which cannot be captured: capture
    // on the private stream, launch on the caller's
    TM_CUDA_CHECK(cudaStreamSynchronize(c.stream));
    cudaStream_t saved = c.stream;
    c.stream = c.capStream;
    const long long n0 = launch_count();
    cudaGraph_t g = nullptr;
    TM_CUDA_CHECK(cudaStreamBeginCapture(c.capStream, cudaStreamCaptureModeThreadLocal));
    try {
      vcycle<T>(c, r, z);
    } catch (...) {
      cudaStreamEndCapture(c.capStream, &g);
      if (g) cudaGraphDestroy(g);
      c.stream = saved;
      throw;
    }
    c.stream = saved;
    TM_CUDA_CHECK(cudaStreamEndCapture(c.capStream, &g));
    c.vcNodes[idx] = launch_count() - n0;
    note_launch((int)-c.vcNodes[idx]);   // captured, not run
    const cudaError_t e = cudaGraphInstantiate(&c.vcGraph[idx], g, 0);
    cudaGraphDestroy(g);
    TM_CUDA_CHECK(e);
    c.vcKey[idx] = key;
  }
  TM_CUDA_CHECK(cudaGraphLaunch(c.vcGraph[idx], c.stream));
  note_launch((int)c.vcNodes[idx]);
}

// Launch-shape autotuner of the FP32 V-cycle, run once per hierarchy before the cycle is first
// captured: per shell level the warps per block (2, 4 or 8) of the column sweep and of the
// residual kernel, and the stage count (2 or 3) of the TMA level-0 sweep. Each candidate is
// timed with events over ten launches on scratch vectors (the kernels' memory traffic and
// arithmetic do not depend on the values); a candidate replaces the default (4 warps, the
// planner's stage count) only when it is at least 3 % faster, so that timing noise does not
// move the shapes. Shapes the caller pinned are applied without timing.
void autotune_vcycle32(Context& c) {
  if (c.tunedEpoch == c.structEpoch) return;
  c.shapeEpoch++;
  std::vector<ShellLevel*> swept;
  for (auto* Lp : c.shells)
    if (!Lp->coarsest && Lp->colorCount[0]) swept.push_back(Lp);
  if (c.shapesPinned) {
    for (size_t k = 0; k < swept.size(); k++) {
      swept[k]->wpbSweep = k < c.pinSweep.size() ? c.pinSweep[k] : 4;
      swept[k]->wpbApply = k < c.pinApply.size() ? c.pinApply[k] : 4;
    }
    c.tsStages = c.pinStages >= 2 && c.pinStages <= c.tsPlanned && sweep_tma_smem(c.tsMaxNodes, c.pinStages) != ~(size_t)0 ? c.pinStages
                                                                                                                              : c.tsPlanned;
    c.tunedEpoch = c.structEpoch;
    return;
  }
  cudaStream_t st = c.stream;
  cudaEvent_t ea, eb;
  TM_CUDA_CHECK(cudaEventCreate(&ea));
  TM_CUDA_CHECK(cudaEventCreate(&eb));
  int smemMax = 0;
  TM_CUDA_CHECK(cudaDeviceGetAttribute(&smemMax, cudaDevAttrMaxSharedMemoryPerBlockOptin, c.dev));
  const int reps = 10;
  auto timed = [&](auto&& launch) {
    launch();
    TM_CUDA_CHECK(cudaEventRecord(ea, st));
    for (int q = 0; q < reps; q++) launch();
    TM_CUDA_CHECK(cudaEventRecord(eb, st));
    TM_CUDA_CHECK(cudaEventSynchronize(eb));
    note_launch(reps + 1);
    float ms = 0;
    TM_CUDA_CHECK(cudaEventElapsedTime(&ms, ea, eb));
    TM_CUDA_CHECK(cudaGetLastError());
    return 1000.0 * ms / reps;
  };
  const int cands[3] = {4, 2, 8};   // the default first
  for (ShellLevel* Lp : swept) {
    ShellLevel& L = *Lp;
    const bool sai = shell_stage_ai<float>(L.maxm);
    const size_t per = shell_sweep_bytes<float>(L.maxm, L.maxColBlocks, sai);
    DBuf<float> sx, sb, sr;
    sx.alloc(6 * (size_t)L.nn); sx.zero(st);
    sb.alloc(6 * (size_t)L.nn); sb.zero(st);
    sr.alloc(6 * (size_t)L.nn);
    L.wpbSweep = L.wpbApply = 4;
    double bestS = 1e30, bestA = 1e30;
    for (int wpb : cands) {
      const size_t smem = wpb * per;
      if (smem > (size_t)smemMax) continue;
      const int attr = (int)std::max<size_t>(smem, 48 * 1024);
      TM_CUDA_CHECK(cudaFuncSetAttribute(k_sweep_shell<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, attr));
      TM_CUDA_CHECK(cudaFuncSetAttribute(k_apply_shell<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, attr));
      const double tS = timed([&] {
        k_sweep_shell<float><<<grid_for(L.colorCount[0], wpb), 32 * wpb, smem, st>>>(L.colorCount[0], L.d_colorMeta[0].p,
            (const long long*)L.d_colorCf[0].p, L.d_rowPtr.p, L.d_col.p, L.d_val32.p, L.d_cfInv32.p, sb.p, sx.p, L.maxm, L.maxColBlocks, 0,
            sai ? 1 : 0);
      });
      const int ncol = L.nx * L.ny;
      const double tA = timed([&] {
        k_apply_shell<float><<<grid_for(ncol, wpb), 32 * wpb, smem, st>>>(ncol, L.d_colMeta.p, L.d_rowPtr.p, L.d_col.p, L.d_val32.p, sx.p,
                                                                           sb.p, sr.p, L.maxm, L.maxColBlocks);
      });
      if (tS < 0.97 * bestS) { bestS = tS; L.wpbSweep = wpb; }
      if (tA < 0.97 * bestA) { bestA = tA; L.wpbApply = wpb; }
    }
  }
  if (c.tsReady && c.colorCount[0] && !c.mf) {
    const size_t n = 3 * (size_t)c.nn;
    DBuf<float> sx, sb;
    sx.alloc(n); sx.zero(st);
    sb.alloc(n); sb.zero(st);
    int best = c.tsPlanned;
    double bestT = 1e30;
    for (int ns = c.tsPlanned; ns >= 2; ns--) {   // the planner's count first
      if (sweep_tma_smem(c.tsMaxNodes, ns) == ~(size_t)0) continue;
      c.tsStages = ns;
      const double t = timed([&] { launch_sweep_tma(c, 0, 0, sb.p, sx.p); });
      if (t < 0.97 * bestT) { bestT = t; best = ns; }
    }
    c.tsStages = best;
  }
  TM_CUDA_CHECK(cudaEventDestroy(ea));
  TM_CUDA_CHECK(cudaEventDestroy(eb));
  TM_CUDA_CHECK(cudaStreamSynchronize(st));
  check_device_error(c);
  c.tunedEpoch = c.structEpoch;
}

void launch_vcycle(Context& c, const double* r, double* z, bool mixed) {
  (void)mixed;
  vcycle_graph<double>(c, r, z);
}

void launch_vcycle32(Context& c, const float* r, float* z) {
  autotune_vcycle32(c);
  vcycle_graph<float>(c, r, z);
}

}  // namespace tmg
