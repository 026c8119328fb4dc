// IC(0) preconditioner of the scaled level-0 operator on the GPU: the fallback of the solve
// policy (LinearSolver.solve, src/core/10-solver.js:967-976) and a preferred kind of its own.
//
// Follows src/core/10-solver.js:
//   scalarUpperCSR   :719-737  scalar upper CSR of the block pattern, sorted columns
//   ICPC.build       :750-761  Manteuffel shift: diag *= 1 + shift, shift 0, 1e-3, x10 .. 1
//   ICPC._factor     :762-782  row-by-row factorization with merge-walk updates
//   ICPC.apply       :784-798  forward (column scatter) and backward (row gather) solves
//
// The reference factors and solves row by row. Here every row gathers the updates it receives,
// in ascending order of the rows they come from (the reference's outer loop order), so each
// entry sees the same subtractions in the same order: the factor and the applied
// preconditioner are bit-identical to the reference's. Rows run in node level sets: a node's
// three rows in one warp, after every node with a lower id that shares a block with it
// (factorization, forward solve) or with a higher id (backward solve). The lanes fetch the
// operands and form the products in parallel; the sums run in the reference's order. Compiled
// without fused multiply-add.
#include <algorithm>
#include <cmath>
#include <vector>

#include "tm_internal.h"

namespace tmg {

namespace {

constexpr double IC_SHIFT0 = 1e-3;     // 00-constants.js:83-84
constexpr double IC_SHIFT_MAX = 1;

inline int grid_for(size_t n, int block) { return (int)((n + block - 1) / block); }

// U0: the operator's values at the scalar upper entries, the diagonal times 1 + shift
__global__ void k_ic_gather(int n, const int* __restrict__ rowPtr, const int* __restrict__ gmap, const double* __restrict__ val,
                            double shift, double* __restrict__ U) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= n) return;
  const int kb = rowPtr[r], ke = rowPtr[r + 1];
  for (int k = kb; k < ke; k++) U[k] = val[gmap[k]];
  if (shift > 0) U[kb] *= 1 + shift;
}

constexpr int IC_WARPS = 4;             // nodes (warps) per block
constexpr int IC_ROWMAX = 64;           // longest scalar row of U (13 upper neighbours x 3 + 3 = 42)
constexpr unsigned FULL = 0xffffffffu;

// one level of the factorization: warp per node, its rows 3n, 3n+1, 3n+2 in order. The row
// being factored sits in shared memory; for every row i < r with U(i, r) != 0, in ascending i,
// the lanes take row i's entries from (i, r) on and subtract U(i, r) U(i, j2) from the entry
// (r, j2) they match (distinct entries per lane; a warp barrier between consecutive i keeps every
// entry's subtractions in ascending i).
__global__ void __launch_bounds__(32 * IC_WARPS) k_ic_factor(int cnt, const int* __restrict__ nodes, const int* __restrict__ rowPtr,
                                                           const int* __restrict__ col, const int* __restrict__ tStart,
                                                           const int* __restrict__ tRow, const int* __restrict__ tPos,
                                                           double* __restrict__ U, int* __restrict__ fail) {
  __shared__ double sVal[IC_WARPS][IC_ROWMAX];
  __shared__ int sCol[IC_WARPS][IC_ROWMAX];
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int t = blockIdx.x * IC_WARPS + w;
  if (t >= cnt) return;
  const int node = nodes[t];
  double* rv = sVal[w];
  int* rc = sCol[w];
  for (int p = 0; p < 3; p++) {
    const int r = 3 * node + p;
    const int kb = rowPtr[r], len = rowPtr[r + 1] - kb;   // len <= IC_ROWMAX (checked on the host)
    for (int e = lane; e < len; e += 32) { rv[e] = U[kb + e]; rc[e] = col[kb + e]; }
    __syncwarp();
    const int q0 = tStart[r], q1 = tStart[r + 1];
    for (int qb = q0; qb < q1; qb += 32) {
      // the next (up to) 32 source rows, fetched in parallel
      int mi = 0, mk = 0, mend = 0;
      double mu = 0;
      if (qb + lane < q1) { mi = tRow[qb + lane]; mk = tPos[qb + lane]; mu = U[mk]; mend = rowPtr[mi + 1]; }
      const int m = min(32, q1 - qb);
      for (int l = 0; l < m; l++) {
        const int kij = __shfl_sync(FULL, mk, l), iend = __shfl_sync(FULL, mend, l);
        const double u1 = __shfl_sync(FULL, mu, l);
        for (int k2 = kij + lane; k2 < iend; k2 += 32) {
          const int j2 = col[k2];
          int lo = 0, hi = len - 1;          // the entry (r, j2), if any: binary search of the sorted row
          while (lo < hi) { const int mid = (lo + hi) >> 1; if (rc[mid] < j2) lo = mid + 1; else hi = mid; }
          if (rc[lo] == j2) rv[lo] -= u1 * U[k2];
        }
        __syncwarp();
      }
    }
    const double d = rv[0];
    if (!(d > 0)) {   // not positive definite at this shift: the attempt fails
      if (lane == 0) atomicExch(fail, 1);
      return;
    }
    const double uii = sqrt(d);
    for (int e = lane; e < len; e += 32) U[kb + e] = e == 0 ? uii : rv[e] / uii;
    __syncwarp();
  }
}

// one level of the forward solve U^T y = b: warp per node; y(r) = (b(r) - sum_i U(i, r) y(i)) / U(r, r)
// with the products formed in parallel and subtracted in ascending i by every lane alike
__global__ void __launch_bounds__(32 * IC_WARPS) k_ic_forward(int cnt, const int* __restrict__ nodes, const int* __restrict__ rowPtr,
                                                            const int* __restrict__ tStart, const int* __restrict__ tRow,
                                                            const int* __restrict__ tPos, const double* __restrict__ U,
                                                            const double* b, double* y) {
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int t = blockIdx.x * IC_WARPS + w;
  if (t >= cnt) return;
  const int node = nodes[t];
  for (int p = 0; p < 3; p++) {
    const int r = 3 * node + p;
    double s = b[r];
    const int q0 = tStart[r], q1 = tStart[r + 1];
    for (int qb = q0; qb < q1; qb += 32) {
      const int q = qb + lane;
      const double prod = q < q1 ? U[tPos[q]] * y[tRow[q]] : 0.0;
      const int m = min(32, q1 - qb);
      for (int l = 0; l < m; l++) s -= __shfl_sync(FULL, prod, l);
    }
    const double yr = s / U[rowPtr[r]];
    __syncwarp();                        // every lane has read b(r) (b may be y)
    if (lane == 0) y[r] = yr;
    __syncwarp();
  }
}

// one level of the backward solve U z = y in place: warp per node, rows 3n+2, 3n+1, 3n
__global__ void __launch_bounds__(32 * IC_WARPS) k_ic_backward(int cnt, const int* __restrict__ nodes, const int* __restrict__ rowPtr,
                                                             const int* __restrict__ col, const double* __restrict__ U, double* z) {
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int t = blockIdx.x * IC_WARPS + w;
  if (t >= cnt) return;
  const int node = nodes[t];
  for (int p = 2; p >= 0; p--) {
    const int r = 3 * node + p;
    const int kb = rowPtr[r], ke = rowPtr[r + 1];
    double s = z[r];
    for (int base = kb + 1; base < ke; base += 32) {
      const int k = base + lane;
      const double prod = k < ke ? U[k] * z[col[k]] : 0.0;
      const int m = min(32, ke - base);
      for (int l = 0; l < m; l++) s -= __shfl_sync(FULL, prod, l);
    }
    const double zr = s / U[kb];
    __syncwarp();
    if (lane == 0) z[r] = zr;
    __syncwarp();
  }
}

// node level sets of a node pattern (rowPtr/col over nodes, sorted): level[i] = 1 + max level
// of the neighbours on the given side (lower or higher ids), grouped by a counting sort;
// start[l] .. start[l+1]-1 index the level's nodes
void level_sets(int nn, const std::vector<int>& nrp, const std::vector<int>& ncol, bool lower, std::vector<int>& nodes,
                std::vector<int>& start) {
  std::vector<int> lev(nn, 0);
  int maxLev = 0;
  auto visit = [&](int i) {
    int l = 0;
    for (int k = nrp[i]; k < nrp[i + 1]; k++) {
      const int j = ncol[k];
      if (lower ? j < i : j > i) l = std::max(l, lev[j] + 1);
    }
    lev[i] = l;
    maxLev = std::max(maxLev, l);
  };
  if (lower) for (int i = 0; i < nn; i++) visit(i);
  else for (int i = nn - 1; i >= 0; i--) visit(i);
  start.assign(maxLev + 2, 0);
  for (int i = 0; i < nn; i++) start[lev[i] + 1]++;
  for (int l = 0; l <= maxLev; l++) start[l + 1] += start[l];
  nodes.assign(nn, 0);
  std::vector<int> fill(start.begin(), start.end() - 1);
  for (int i = 0; i < nn; i++) nodes[fill[lev[i]]++] = i;
}

}  // namespace

// scalarUpperCSR (10-solver.js:719-737) of a node pattern: nrp/ncol the sorted block columns of
// every node, vbase[k] the index of block k's (0, 0) value and vstride the step between its
// nine values (component 3p + q at vbase[k] + vstride (3p + q))
void ic_build_structure(IcFactor& F, int nn, const std::vector<int>& nrp, const std::vector<int>& ncol,
                        const std::vector<long long>& vbase, long long vstride, cudaStream_t st) {
  const int n = 3 * nn;
  std::vector<int> rowPtr(n + 1, 0);
  for (int i = 0; i < nn; i++) {
    int up = 0;
    bool diag = false;
    for (int k = nrp[i]; k < nrp[i + 1]; k++) {
      if (ncol[k] > i) up++;
      else if (ncol[k] == i) diag = true;
    }
    if (!diag) fail(TM_BAD_INPUT, "IC(0): a node without its diagonal block");
    for (int p = 0; p < 3; p++) rowPtr[3 * i + p + 1] = rowPtr[3 * i + p] + 3 * up + (3 - p);
  }
  const long long nnz = rowPtr[n];
  for (int r = 0; r < n; r++)
    if (rowPtr[r + 1] - rowPtr[r] > IC_ROWMAX) fail(TM_BAD_INPUT, "IC(0): a scalar row longer than the factor kernel holds");
  std::vector<int> col(nnz), gmap(nnz);
  std::vector<int> tCount(n + 1, 0);
  for (int i = 0; i < nn; i++)
    for (int p = 0; p < 3; p++) {
      int w = rowPtr[3 * i + p];
      for (int k = nrp[i]; k < nrp[i + 1]; k++) {
        const int j = ncol[k];
        if (j < i) continue;
        for (int q = (j == i ? p : 0); q < 3; q++) {
          const long long g = vbase[k] + vstride * (3 * p + q);
          if (g >= (1LL << 31)) fail(TM_BAD_INPUT, "IC(0): operator too large for 32-bit entry indices");
          col[w] = 3 * j + q;
          gmap[w] = (int)g;
          if (w > rowPtr[3 * i + p]) tCount[3 * j + q + 1]++;
          w++;
        }
      }
    }
  for (int r = 0; r < n; r++) tCount[r + 1] += tCount[r];
  std::vector<int> tRow(tCount[n]), tPos(tCount[n]);
  std::vector<int> fill(tCount.begin(), tCount.end() - 1);
  for (int r = 0; r < n; r++)        // rows ascending: every column list comes out in ascending row order
    for (int k = rowPtr[r] + 1; k < rowPtr[r + 1]; k++) {
      const int cc = col[k];
      tRow[fill[cc]] = r;
      tPos[fill[cc]] = k;
      fill[cc]++;
    }
  std::vector<int> fwd, fwdStart, bwd, bwdStart;
  level_sets(nn, nrp, ncol, true, fwd, fwdStart);
  level_sets(nn, nrp, ncol, false, bwd, bwdStart);
  F.d_rowPtr.upload(rowPtr, st); F.d_col.upload(col, st); F.d_gmap.upload(gmap, st);
  F.d_tStart.upload(tCount, st); F.d_tRow.upload(tRow, st); F.d_tPos.upload(tPos, st);
  F.d_fwdNodes.upload(fwd, st); F.d_bwdNodes.upload(bwd, st);
  F.fwdStart = fwdStart; F.bwdStart = bwdStart;
  F.drop_graph();
  F.d_U.alloc(nnz);
  F.d_fail.alloc(1);
  F.n = n; F.nnz = nnz;
  F.ready = false;
  TM_CUDA_CHECK(cudaStreamSynchronize(st));
}

// ICPC.build (10-solver.js:750-761): factor of the values val (gathered through the structure's
// map) with the shift sequence 0, 1e-3, 1e-2, ... 1
void ic_factor(IcFactor& F, const double* val, cudaStream_t st) {
  F.ready = false;
  double shift = 0;
  for (int attempt = 0; attempt < 8; attempt++) {
    F.d_fail.zero(st);
    note_launch();
    k_ic_gather<<<grid_for(F.n, 256), 256, 0, st>>>(F.n, F.d_rowPtr.p, F.d_gmap.p, val, shift, F.d_U.p);
    TM_CUDA_CHECK(cudaGetLastError());
    const int nl = (int)F.fwdStart.size() - 1;
    for (int l = 0; l < nl; l++) {
      const int cnt = F.fwdStart[l + 1] - F.fwdStart[l];
      if (cnt <= 0) continue;
      note_launch();
      k_ic_factor<<<grid_for(cnt, IC_WARPS), 32 * IC_WARPS, 0, st>>>(cnt, F.d_fwdNodes.p + F.fwdStart[l], F.d_rowPtr.p, F.d_col.p,
                                                                    F.d_tStart.p, F.d_tRow.p, F.d_tPos.p, F.d_U.p, F.d_fail.p);
    }
    TM_CUDA_CHECK(cudaGetLastError());
    int bad = 0;
    TM_CUDA_CHECK(cudaMemcpyAsync(&bad, F.d_fail.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    TM_CUDA_CHECK(cudaStreamSynchronize(st));
    if (!bad) { F.shift = shift; F.ready = true; return; }
    shift = shift == 0 ? IC_SHIFT0 : shift * 10;
    if (shift > IC_SHIFT_MAX) shift = IC_SHIFT_MAX;
  }
  fail(TM_BAD_INPUT, "IC(0) failed even with the maximum diagonal shift");
}

namespace {
void ic_apply_launches(IcFactor& F, const double* r, double* z, cudaStream_t st) {
  const int nl = (int)F.fwdStart.size() - 1, nb = (int)F.bwdStart.size() - 1;
  for (int l = 0; l < nl; l++) {
    const int cnt = F.fwdStart[l + 1] - F.fwdStart[l];
    if (cnt <= 0) continue;
    k_ic_forward<<<grid_for(cnt, IC_WARPS), 32 * IC_WARPS, 0, st>>>(cnt, F.d_fwdNodes.p + F.fwdStart[l], F.d_rowPtr.p, F.d_tStart.p,
                                                                   F.d_tRow.p, F.d_tPos.p, F.d_U.p, r, z);
  }
  for (int l = 0; l < nb; l++) {
    const int cnt = F.bwdStart[l + 1] - F.bwdStart[l];
    if (cnt <= 0) continue;
    k_ic_backward<<<grid_for(cnt, IC_WARPS), 32 * IC_WARPS, 0, st>>>(cnt, F.d_bwdNodes.p + F.bwdStart[l], F.d_rowPtr.p, F.d_col.p,
                                                                    F.d_U.p, z);
  }
}
}  // namespace

// ICPC.apply (10-solver.js:784-798): the level launches, replayed from a CUDA graph captured on
// the first apply with these vectors on this stream (a created stream; the legacy default stream
// launches directly). The factor is updated in place, so the graph stays valid until the
// structure changes.
void ic_apply(IcFactor& F, const double* r, double* z, cudaStream_t st) {
  if (!F.ready) fail(TM_BAD_INPUT, "IC(0) preconditioner not built");
  const int nl = (int)F.fwdStart.size() - 1, nb = (int)F.bwdStart.size() - 1;
  note_launch(nl + nb);
  if (st == nullptr || st == cudaStreamLegacy || st == cudaStreamPerThread) {
    ic_apply_launches(F, r, z, st);
    TM_CUDA_CHECK(cudaGetLastError());
    return;
  }
  if (!F.exec || F.gr != r || F.gz != z || F.gst != st) {
    F.drop_graph();
    cudaGraph_t g = nullptr;
    TM_CUDA_CHECK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    ic_apply_launches(F, r, z, st);
    const cudaError_t le = cudaGetLastError();
    TM_CUDA_CHECK(cudaStreamEndCapture(st, &g));
    if (le != cudaSuccess) { cudaGraphDestroy(g); TM_CUDA_CHECK(le); }
    const cudaError_t ie = cudaGraphInstantiate(&F.exec, g, 0);
    cudaGraphDestroy(g);
    TM_CUDA_CHECK(ie);
    F.gr = r; F.gz = z; F.gst = st;
  }
  TM_CUDA_CHECK(cudaGraphLaunch(F.exec, st));
}

// the level-0 operator of a solve context: node pattern from the stencil slots (ascending
// neighbour ids), values in the slot-major operator
void build_ic(Context& c) {
  IcFactor& F = c.ic;
  if (F.epoch != c.structEpoch || F.n != 3 * c.nn) {
    const int nn = c.nn;
    std::vector<int> nrp(nn + 1, 0), ncol;
    std::vector<long long> vbase;
    for (int i = 0; i < nn; i++) {
      for (int s = 0; s < NSLOT; s++) {
        if (!(c.slotMask[i] >> s & 1)) continue;
        ncol.push_back(c.nbr[(size_t)s * nn + i]);
        vbase.push_back((long long)s * 9 * c.nnp + c.pos[i]);
      }
      nrp[i + 1] = (int)ncol.size();
    }
    ic_build_structure(F, nn, nrp, ncol, vbase, c.nnp, c.stream);
    F.epoch = c.structEpoch;
  }
  ic_factor(F, c.d_val.p, c.stream);
}

void launch_ic_apply(Context& c, const double* r, double* z) { ic_apply(c.ic, r, z, c.stream); }

}  // namespace tmg
