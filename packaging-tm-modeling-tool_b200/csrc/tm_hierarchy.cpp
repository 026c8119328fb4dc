// Host-side structure of the device model: node stencils, element classes and the
// multigrid hierarchy (aggregates, prolongation sparsity and geometric weights,
// Galerkin patterns). The structure depends only on the mesh, so it is built once
// per context; all numeric set-up (assembly, scaling, factors, Galerkin values) runs
// on the GPU every step.
//
// The hierarchy follows the reference's MultigridPC (src/core/10-solver.js:620-650):
//   buildShellLevel        :260-334   solid level -> shell aggregates (6 DOFs)
//   coarseLines            :171-177   x-y semi-coarsening keeping feature lines
//   buildCoarseShellLevel  :396-471   Hermite / linear interpolation with rbmShift
//   galerkinProduct        :193-245   (pattern part: sorted touched coarse columns)
//   factorCoarsest         :562-566   band width of the coarsest operator
#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <set>
#include <tuple>

#include "tm_internal.h"

namespace tmg {

namespace {

// compliant parts (10-solver.js:248): SOLDER 1, UF_BUMP 2, UF_FILLET 3, TIM 5, LIDADH 7, STIFFADH 9
bool compliant_part(int p) { return p == 1 || p == 2 || p == 3 || p == 5 || p == 7 || p == 9; }

const int LOC[8][3] = {{0, 0, 0}, {1, 0, 0}, {1, 1, 0}, {0, 1, 0}, {0, 0, 1}, {1, 0, 1}, {1, 1, 1}, {0, 1, 1}};

std::vector<int> coarse_lines(int n, const std::vector<int>* keep) {
  std::set<int> s;
  for (int i = 0; i < n; i += 2) s.insert(i);
  s.insert(n - 1);
  if (keep) for (int k : *keep) if (k >= 0 && k < n) s.insert(k);
  return std::vector<int>(s.begin(), s.end());
}

void hermite_pair(double t, double h, bool alongY, double* WA, double* WB) {
  std::fill(WA, WA + 36, 0.0);
  std::fill(WB, WB + 36, 0.0);
  for (int d = 0; d < 6; d++) { WA[d * 6 + d] = 1 - t; WB[d * 6 + d] = t; }
  const double h00 = 2 * t * t * t - 3 * t * t + 1, h10 = t * t * t - 2 * t * t + t, h01 = -2 * t * t * t + 3 * t * t, h11 = t * t * t - t * t;
  WA[2 * 6 + 2] = h00; WB[2 * 6 + 2] = h01;
  if (alongY) { WA[2 * 6 + 3] = h * h10; WB[2 * 6 + 3] = h * h11; }
  else { WA[2 * 6 + 4] = -h * h10; WB[2 * 6 + 4] = -h * h11; }
}

void rbm_shift(double dz, double* M) {
  std::fill(M, M + 36, 0.0);
  for (int d = 0; d < 6; d++) M[d * 7] = 1;
  M[0 * 6 + 4] = dz; M[1 * 6 + 3] = -dz; M[2 * 6 + 5] = dz;
}

void mul66(const double* A, const double* B, double* C) {
  double T[36];
  for (int i = 0; i < 6; i++)
    for (int j = 0; j < 6; j++) {
      double s = 0;
      for (int k = 0; k < 6; k++) s += A[i * 6 + k] * B[k * 6 + j];
      T[i * 6 + j] = s;
    }
  std::memcpy(C, T, sizeof(T));
}

int match_aggregate(const ShellLevel& C, int col, double zlo, double zhi, double zref) {
  int best = -1;
  double bo = 0;
  for (int a = C.colStart[col]; a < C.colStart[col + 1]; a++) {
    const double ov = std::min(zhi, C.zhi[a]) - std::max(zlo, C.zlo[a]);
    const double score = ov > 0 ? ov + 1e-9 : (zref >= C.zlo[a] - 1e-9 && zref <= C.zhi[a] + 1e-9 ? 1e-9 : -1);
    if (score > bo) { bo = score; best = a; }
  }
  return best;
}

void color_lists(int nx, int ny, const std::vector<int>& colStart, DBuf<int>* d_lists, int* counts, cudaStream_t s) {
  std::vector<int> lists[4];
  for (int c = 0; c < nx * ny; c++) {
    if (colStart[c + 1] == colStart[c]) continue;
    const int i = c / ny, j = c % ny;
    lists[(i & 1) * 2 + (j & 1)].push_back(c);
  }
  for (int k = 0; k < 4; k++) {
    counts[k] = (int)lists[k].size();
    d_lists[k].upload(lists[k], s);
  }
}

// Galerkin pattern of a shell level from its fine level (sorted touched columns per coarse row)
void galerkin_pattern_shell(const ShellLevel& F, ShellLevel& C) {
  const int nnc = C.nn;
  std::vector<int> mark(nnc, -1), touched;
  C.rowPtr.assign(nnc + 1, 0);
  C.col.clear();
  int maxr = 0;
  for (int I = 0; I < nnc; I++) {
    touched.clear();
    for (int q = F.chPtr[I]; q < F.chPtr[I + 1]; q++) {
      const int f = F.chIdx[q];
      for (int k = F.rowPtr[f]; k < F.rowPtr[f + 1]; k++) {
        const int g = F.col[k];
        for (int p = F.prolPtr[g]; p < F.prolPtr[g + 1]; p++) {
          const int J = F.prolIdx[p];
          if (mark[J] != I) { mark[J] = I; touched.push_back(J); }
        }
      }
    }
    std::sort(touched.begin(), touched.end());
    C.rowPtr[I + 1] = C.rowPtr[I] + (int)touched.size();
    C.col.insert(C.col.end(), touched.begin(), touched.end());
    maxr = std::max(maxr, (int)touched.size());
  }
  C.nb = (int)C.col.size();
  C.maxRowBlocks = maxr;
  C.diag.assign(nnc, 0);
  for (int I = 0; I < nnc; I++)
    for (int k = C.rowPtr[I]; k < C.rowPtr[I + 1]; k++)
      if (C.col[k] == I) { C.diag[I] = k; break; }
}

void transpose_prol(ShellLevel& F, int nnc) {
  F.chPtr.assign(nnc + 1, 0);
  for (size_t q = 0; q < F.prolIdx.size(); q++) F.chPtr[F.prolIdx[q] + 1]++;
  for (int c = 0; c < nnc; c++) F.chPtr[c + 1] += F.chPtr[c];
  F.chIdx.assign(F.prolIdx.size(), 0);
  F.chW.assign(F.prolIdx.size(), 0);
  std::vector<int> fill(F.chPtr.begin(), F.chPtr.begin() + nnc);
  for (int f = 0; f < F.nn; f++)
    for (int q = F.prolPtr[f]; q < F.prolPtr[f + 1]; q++) {
      const int c = F.prolIdx[q];
      F.chIdx[fill[c]] = f;
      F.chW[fill[c]] = q;
      fill[c]++;
    }
}

// buildCoarseShellLevel (10-solver.js:396-471): structure of the coarse level C, and the
// prolongation from C to L (parents with geometric 6x6 weights) with its transpose
ShellLevel* build_coarse_shell(ShellLevel& L) {
  const std::vector<int> cx = coarse_lines(L.nx, L.hasKeep ? &L.keepX : nullptr);
  const std::vector<int> cy = coarse_lines(L.ny, L.hasKeep ? &L.keepY : nullptr);
  const int nxc = (int)cx.size(), nyc = (int)cy.size();
  ShellLevel* Cp = new ShellLevel();
  ShellLevel& C = *Cp;
  C.nx = nxc; C.ny = nyc;
  C.xs.resize(nxc); C.ys.resize(nyc);
  for (int I = 0; I < nxc; I++) C.xs[I] = L.xs[cx[I]];
  for (int J = 0; J < nyc; J++) C.ys[J] = L.ys[cy[J]];
  C.colStart.assign((size_t)nxc * nyc + 1, 0);
  int na = 0;
  for (int I = 0; I < nxc; I++)
    for (int J = 0; J < nyc; J++) {
      C.colStart[I * nyc + J] = na;
      const int col = cx[I] * L.ny + cy[J];
      for (int a = L.colStart[col]; a < L.colStart[col + 1]; a++) {
        C.zlo.push_back(L.zlo[a]); C.zhi.push_back(L.zhi[a]); C.zref.push_back(L.zref[a]);
        na++;
      }
    }
  C.colStart[(size_t)nxc * nyc] = na;
  C.nn = na;
  C.hasKeep = L.hasKeep;
  if (L.hasKeep) {
    for (int i : L.keepX) { auto it = std::find(cx.begin(), cx.end(), i); if (it != cx.end()) C.keepX.push_back((int)(it - cx.begin())); }
    for (int j : L.keepY) { auto it = std::find(cy.begin(), cy.end(), j); if (it != cy.end()) C.keepY.push_back((int)(it - cy.begin())); }
  }
  struct Loc { int I0, I1; double t, h; };
  auto locate = [](const std::vector<int>& lines, const std::vector<double>& coords, int i, double x) {
    int I0 = 0;
    while (I0 + 1 < (int)lines.size() && lines[I0 + 1] <= i) I0++;
    if (lines[I0] == i) return Loc{I0, -1, 0, 0};
    return Loc{I0, I0 + 1, (x - coords[I0]) / (coords[I0 + 1] - coords[I0]), coords[I0 + 1] - coords[I0]};
  };
  L.prolPtr.assign(L.nn + 1, 0);
  L.prolIdx.clear();
  L.prolW.clear();
  double WL[36], WR[36], WB[36], WT[36], tmp[36], sh[36], tmp2[36];
  for (int i = 0; i < L.nx; i++) {
    const Loc px = locate(cx, C.xs, i, L.xs[i]);
    for (int j = 0; j < L.ny; j++) {
      const Loc py = locate(cy, C.ys, j, L.ys[j]);
      const int col = i * L.ny + j;
      for (int f = L.colStart[col]; f < L.colStart[col + 1]; f++) {
        auto get = [&](int I, int J) { return match_aggregate(C, I * nyc + J, L.zlo[f], L.zhi[f], L.zref[f]); };
        std::vector<int> xC = px.I1 < 0 ? std::vector<int>{px.I0} : std::vector<int>{px.I0, px.I1};
        std::vector<int> yC = py.I1 < 0 ? std::vector<int>{py.I0} : std::vector<int>{py.I0, py.I1};
        std::map<std::pair<int, int>, int> par;
        bool complete = true;
        for (int I : xC) for (int J : yC) { const int a = get(I, J); par[{I, J}] = a; if (a < 0) complete = false; }
        int count = 0;
        auto push = [&](int I, int J, const double* W) {
          const int a = par[{I, J}];
          rbm_shift(L.zref[f] - C.zref[a], sh);
          mul66(W, sh, tmp2);
          L.prolIdx.push_back(a);
          L.prolW.insert(L.prolW.end(), tmp2, tmp2 + 36);
          count++;
        };
        if (complete) {
          if (px.I1 >= 0) hermite_pair(px.t, px.h, false, WL, WR);
          if (py.I1 >= 0) hermite_pair(py.t, py.h, true, WB, WT);
          if (px.I1 < 0 && py.I1 < 0) { double W[36] = {0}; for (int d = 0; d < 6; d++) W[d * 7] = 1; push(px.I0, py.I0, W); }
          else if (py.I1 < 0) { push(px.I0, py.I0, WL); push(px.I1, py.I0, WR); }
          else if (px.I1 < 0) { push(px.I0, py.I0, WB); push(px.I0, py.I1, WT); }
          else {
            mul66(WB, WL, tmp); push(px.I0, py.I0, tmp); mul66(WB, WR, tmp); push(px.I1, py.I0, tmp);
            mul66(WT, WL, tmp); push(px.I0, py.I1, tmp); mul66(WT, WR, tmp); push(px.I1, py.I1, tmp);
          }
        } else {
          const std::vector<double> wx = px.I1 < 0 ? std::vector<double>{1} : std::vector<double>{1 - px.t, px.t};
          const std::vector<double> wy = py.I1 < 0 ? std::vector<double>{1} : std::vector<double>{1 - py.t, py.t};
          double sum = 0;
          struct Ex { int I, J; double w; };
          std::vector<Ex> ex;
          for (size_t a = 0; a < xC.size(); a++)
            for (size_t b = 0; b < yC.size(); b++) {
              const int ag = par[{xC[a], yC[b]}];
              const double w = wx[a] * wy[b];
              if (ag >= 0 && w > 0) { ex.push_back({xC[a], yC[b], w}); sum += w; }
            }
          for (auto& e : ex) { double W[36] = {0}; for (int d = 0; d < 6; d++) W[d * 7] = e.w / sum; push(e.I, e.J, W); }
        }
        L.prolPtr[f + 1] = count;
      }
    }
  }
  for (int f = 0; f < L.nn; f++) L.prolPtr[f + 1] += L.prolPtr[f];
  transpose_prol(L, na);
  galerkin_pattern_shell(L, C);
  return Cp;
}

// position of coarse column J in the sorted block row I, or -1
int block_of(const ShellLevel& C, int I, int J) {
  const int* b = C.col.data() + C.rowPtr[I];
  const int* e = C.col.data() + C.rowPtr[I + 1];
  const int* q = std::lower_bound(b, e, J);
  return (q != e && *q == J) ? C.rowPtr[I] + (int)(q - b) : -1;
}

// level 0 -> 1 contribution lists (the summands of galerkinProduct, 10-solver.js:193-245, grouped
// by the coarse block they land in); counting sort over (slot, position) keeps that order per block
void galerkin_lists01(Context& c, cudaStream_t st) {
  const ShellLevel& L1 = *c.shells[0];
  const int nn = c.nn;
  std::vector<int> start((size_t)L1.nb + 1, 0);
  auto visit = [&](auto&& emit) {
    for (int s = 0; s < NSLOT; s++)
      for (int ps = 0; ps < nn; ps++) {
        const int i = c.posNode[ps];
        if (!(c.slotMask[i] >> s & 1)) continue;
        const int I = c.nodeAgg[i], J = c.nodeAgg[c.nbr[(size_t)s * nn + i]];
        if (I < 0 || J < 0) continue;   // held nodes have no prolongation
        const int k = block_of(L1, I, J);
        if (k < 0) fail(TM_BAD_INPUT, "level-1 Galerkin pattern misses a stencil coupling");
        emit(k, ps * NSLOT + s);
      }
  };
  visit([&](int k, int) { start[k + 1]++; });
  for (size_t k = 0; k < (size_t)L1.nb; k++) start[k + 1] += start[k];
  std::vector<int> list((size_t)start.back()), fill(start.begin(), start.end() - 1);
  visit([&](int k, int code) { list[fill[k]++] = code; });
  c.d_g01Start.upload(start, st);
  c.d_g01List.upload(list, st);
}

// shell level F -> C contribution lists: (fine block, row weight entry, column weight entry) per
// summand of the 6x6 galerkinProduct, in (coarse row child, fine block, column parent) order
void galerkin_lists_shell(const ShellLevel& F, ShellLevel& C, cudaStream_t st) {
  std::vector<int> start((size_t)C.nb + 1, 0);
  auto visit = [&](auto&& emit) {
    for (int I = 0; I < C.nn; I++)
      for (int q = F.chPtr[I]; q < F.chPtr[I + 1]; q++) {
        const int f = F.chIdx[q];
        for (int k = F.rowPtr[f]; k < F.rowPtr[f + 1]; k++) {
          const int g = F.col[k];
          for (int p = F.prolPtr[g]; p < F.prolPtr[g + 1]; p++) {
            const int b = block_of(C, I, F.prolIdx[p]);
            if (b < 0) fail(TM_BAD_INPUT, "shell Galerkin pattern misses a coupling");
            emit(b, k, F.chW[q], p);
          }
        }
      }
  };
  visit([&](int b, int, int, int) { start[b + 1]++; });
  for (size_t b = 0; b < (size_t)C.nb; b++) start[b + 1] += start[b];
  std::vector<int> list(3 * (size_t)start.back()), fill(start.begin(), start.end() - 1);
  visit([&](int b, int k, int p1, int p2) {
    const size_t t = 3 * (size_t)fill[b]++;
    list[t] = k; list[t + 1] = p1; list[t + 2] = p2;
  });
  C.d_galStart.upload(start, st);
  C.d_galList.upload(list, st);
}

// column metadata of a shell level: aggregate and block ranges of every column, and per colour
// list entry the same plus the offset of the column's inverse (lists in color_lists order)
void shell_column_meta(ShellLevel& L, cudaStream_t st) {
  const int ncol = L.nx * L.ny;
  std::vector<int4> all(ncol);
  std::vector<int4> lists[4];
  std::vector<long long> cfs[4];
  for (int c = 0; c < ncol; c++) {
    const int n0 = L.colStart[c], n1 = L.colStart[c + 1];
    all[c] = make_int4(n0, n1, L.rowPtr[n0], L.rowPtr[n1]);
    if (n1 == n0) continue;
    const int k = ((c / L.ny) & 1) * 2 + ((c % L.ny) & 1);
    lists[k].push_back(all[c]);
    cfs[k].push_back(L.cfPtr.empty() ? 0 : L.cfPtr[c]);
  }
  L.d_colMeta.upload(all, st);
  for (int k = 0; k < 4; k++) {
    L.d_colorMeta[k].upload(lists[k], st);
    L.d_colorCf[k].upload(cfs[k], st);
  }
}

void column_factor_sizes(ShellLevel& L) {
  const int ncol = L.nx * L.ny;
  L.cfPtr.assign(ncol + 1, 0);
  L.maxm = 0;
  for (int col = 0; col < ncol; col++) {
    const int m = (L.colStart[col + 1] - L.colStart[col]) * 6;
    L.cfPtr[col + 1] = L.cfPtr[col] + (long long)m * m;
    L.maxm = std::max(L.maxm, m);
  }
}

}  // namespace

void build_stencil(Context& c) {
  const int nx = c.nx, ny = c.ny, nz = c.nz, nn = c.nn;
  c.nodeIJK.assign(3 * (size_t)nn, 0);
  for (int i = 0; i < nx; i++)
    for (int j = 0; j < ny; j++)
      for (int k = 0; k < nz; k++) {
        const int id = c.nodeId[((size_t)i * ny + j) * nz + k];
        if (id < 0) continue;
        c.nodeIJK[3 * (size_t)id] = i; c.nodeIJK[3 * (size_t)id + 1] = j; c.nodeIJK[3 * (size_t)id + 2] = k;
      }
  c.nbr.assign((size_t)NSLOT * nn, -1);
  for (int n = 0; n < nn; n++) {
    const int i = c.nodeIJK[3 * (size_t)n], j = c.nodeIJK[3 * (size_t)n + 1], k = c.nodeIJK[3 * (size_t)n + 2];
    for (int s = 0; s < NSLOT; s++) {
      const int di = s / 9 - 1, dj = (s / 3) % 3 - 1, dk = s % 3 - 1;
      const int a = i + di, b = j + dj, d = k + dk;
      if (a < 0 || a >= nx || b < 0 || b >= ny || d < 0 || d >= nz) continue;
      c.nbr[(size_t)s * nn + n] = c.nodeId[((size_t)a * ny + b) * nz + d];
    }
  }
  // block pattern (bcsrFromElements + fullPatternFromUpper): nodes sharing an element
  c.slotMask.assign(nn, 0);
  for (int e = 0; e < c.ne; e++)
    for (int a = 0; a < 8; a++)
      for (int b = 0; b < 8; b++) {
        const int s = (LOC[b][0] - LOC[a][0] + 1) * 9 + (LOC[b][1] - LOC[a][1] + 1) * 3 + (LOC[b][2] - LOC[a][2] + 1);
        c.slotMask[c.conn[8 * (size_t)e + a]] |= 1 << s;
      }
  c.maxColLen = 0;
  for (int col = 0; col < nx * ny; col++) c.maxColLen = std::max(c.maxColLen, c.colStart[col + 1] - c.colStart[col]);
  // colour-major positions (colour = (i%2)*2 + j%2 of the column)
  c.pos.assign(nn, -1);
  c.posNode.assign(nn, -1);
  int p = 0;
  for (int k = 0; k < 4; k++)
    for (int col = 0; col < nx * ny; col++) {
      if (((col / ny) & 1) * 2 + ((col % ny) & 1) != k) continue;
      for (int n = c.colStart[col]; n < c.colStart[col + 1]; n++) { c.pos[n] = p; c.posNode[p] = n; p++; }
    }
  if (p != nn) fail(TM_BAD_INPUT, "columns do not cover the nodes");
}

void build_classes(Context& c) {
  std::map<std::tuple<int, double, double, double>, int> key;
  c.eClass.assign(c.ne, 0);
  c.clsPset.clear();
  c.clsH.clear();
  for (int e = 0; e < c.ne; e++) {
    const int i = c.eIJK[3 * (size_t)e], j = c.eIJK[3 * (size_t)e + 1], k = c.eIJK[3 * (size_t)e + 2];
    const double hx = c.xs[i + 1] - c.xs[i], hy = c.ys[j + 1] - c.ys[j], hz = c.zs[k + 1] - c.zs[k];
    auto t = std::make_tuple(c.ePset[e], hx, hy, hz);
    auto it = key.find(t);
    int id;
    if (it == key.end()) {
      id = (int)c.clsPset.size();
      key.emplace(t, id);
      c.clsPset.push_back(c.ePset[e]);
      c.clsH.push_back(hx); c.clsH.push_back(hy); c.clsH.push_back(hz);
    } else {
      id = it->second;
    }
    c.eClass[e] = id;
  }
  c.ncls = (int)c.clsPset.size();
}


// The reference reads cellElems at the flat index (i*ncy + j)*ncz + k for node column (i, j)
// (10-solver.js:270-287); at j = ny-1 that index is cell (i+1, 0, k) and at i = nx-1 it is past
// the array (an undefined entry in JavaScript, i.e. no element). Both are reproduced.
static int cell_elem_at(const Context& c, long cell, int q) {
  const long idx = 2 * cell + q;
  if (idx < 0 || idx >= (long)c.cellElems.size()) return -1;
  return c.cellElems[idx];
}

void build_hierarchy(Context& c) {
  c.structEpoch++;
  const int nx = c.nx, ny = c.ny, nz = c.nz, ncy = ny - 1, ncz = nz - 1, nn = c.nn;
  for (auto* L : c.shells) delete L;
  c.shells.clear();
  // ---- level 1: buildShellLevel (10-solver.js:260-334), mergeSingles 'below' (:626). In a
  // stacked-module stage (c.actElem / c.actNode set, 10-solver.js:262-266) the elements not born in
  // the stage count as void and the nodes they alone touch (held) stay out of every aggregate.
  const bool act = !c.actElem.empty();
  auto elemOn = [&](int e) { return e >= 0 && (!act || c.actElem[e]); };
  ShellLevel* L1 = new ShellLevel();
  L1->nx = nx; L1->ny = ny; L1->xs = c.xs; L1->ys = c.ys;
  L1->colStart.assign((size_t)nx * ny + 1, 0);
  c.nodeAgg.assign(nn, -1);
  auto isCompliant = [&](int i, int j, int k) {
    const long cell = ((long)i * ncy + j) * ncz + k;
    bool any = false, stiff = false;
    for (int q = 0; q < 2; q++) {
      const int e = cell_elem_at(c, cell, q);
      if (!elemOn(e)) continue;
      any = true;
      if (!compliant_part(c.ePart[e])) stiff = true;
    }
    return any && !stiff;
  };
  auto hasElem = [&](int i, int j, int k) {
    const long cell = ((long)i * ncy + j) * ncz + k;
    return elemOn(cell_elem_at(c, cell, 0)) || elemOn(cell_elem_at(c, cell, 1));
  };
  auto elemClass = [&](int i, int j, int k) -> int {
    return (k < 0 || k >= ncz || !hasElem(i, j, k)) ? 0 : (isCompliant(i, j, k) ? 1 : 2);
  };
  int na = 0;
  struct NodeRec { int n; double z; };
  for (int col = 0; col < nx * ny; col++) {
    L1->colStart[col] = na;
    const int i = col / ny, j = col % ny;
    std::vector<std::vector<NodeRec>> runs;
    int cur = -1, prevK = -2, prevType = 0;
    for (int k = 0; k < nz; k++) {
      const int n = c.nodeId[(size_t)col * nz + k];
      if (n < 0 || (act && !c.actNode[n])) { cur = -1; prevK = -2; continue; }
      const int below = elemClass(i, j, k - 1), above = elemClass(i, j, k);
      const int type = (below == 2 || above == 2) ? 2 : 1;
      bool joined = false;
      if (cur >= 0 && prevK == k - 1 && below != 0) joined = below == 2 || (type == 1 && prevType == 1);
      if (!joined) { runs.emplace_back(); cur = (int)runs.size() - 1; }
      runs[cur].push_back({n, c.coords[3 * (size_t)n + 2]});
      prevK = k; prevType = type;
    }
    for (int r = 0; r < (int)runs.size(); r++) {
      if (runs[r].size() != 1 || runs.size() < 2) continue;
      const int t = r > 0 ? r - 1 : r + 1;
      if (t < r) runs[t].push_back(runs[r][0]); else runs[t].insert(runs[t].begin(), runs[r][0]);
      runs.erase(runs.begin() + r);
      r--;
    }
    for (auto& run : runs) {
      double zs = 0;
      for (auto& o : run) { c.nodeAgg[o.n] = na; zs += o.z; }
      L1->zlo.push_back(run[0].z); L1->zhi.push_back(run.back().z); L1->zref.push_back(zs / run.size());
      na++;
    }
  }
  L1->colStart[(size_t)nx * ny] = na;
  L1->nn = na;
  // every node outside the held ones is in exactly one aggregate; the members of aggregate I are
  // aggNodes[aggPtr[I] .. aggPtr[I+1]-1] in ascending node order (a contiguous node range unless held
  // nodes lie between them)
  c.aggPtr.assign(na + 1, 0);
  for (int n = 0; n < nn; n++) {
    const int a = c.nodeAgg[n];
    if (a < 0) {
      if (!act || c.actNode[n]) fail(TM_BAD_INPUT, "node outside every multigrid aggregate");
      continue;
    }
    c.aggPtr[a + 1]++;
  }
  for (int a = 0; a < na; a++) c.aggPtr[a + 1] += c.aggPtr[a];
  c.aggNodes.assign(c.aggPtr[na], 0);
  {
    std::vector<int> fill(c.aggPtr.begin(), c.aggPtr.end() - 1);
    for (int n = 0; n < nn; n++)
      if (c.nodeAgg[n] >= 0) c.aggNodes[fill[c.nodeAgg[n]]++] = n;
  }
  c.zp.assign(nn, 0.0);
  for (int n = 0; n < nn; n++)
    if (c.nodeAgg[n] >= 0) c.zp[n] = c.coords[3 * (size_t)n + 2] - L1->zref[c.nodeAgg[n]];
  L1->hasKeep = !c.featureX.empty() || !c.featureY.empty();
  L1->keepX = c.featureX; L1->keepY = c.featureY;
  // Galerkin pattern 0 -> 1 over the block pattern of the solid level
  {
    std::vector<int> mark(na, -1), touched;
    L1->rowPtr.assign(na + 1, 0);
    int maxr = 0;
    for (int I = 0; I < na; I++) {
      touched.clear();
      for (int q = c.aggPtr[I]; q < c.aggPtr[I + 1]; q++) {
        const int i = c.aggNodes[q];
        const int mask = c.slotMask[i];
        for (int s = 0; s < NSLOT; s++) {
          if (!(mask >> s & 1)) continue;
          const int J = c.nodeAgg[c.nbr[(size_t)s * nn + i]];
          if (J < 0) continue;   // a held neighbour (no prolongation)
          if (mark[J] != I) { mark[J] = I; touched.push_back(J); }
        }
      }
      std::sort(touched.begin(), touched.end());
      L1->rowPtr[I + 1] = L1->rowPtr[I] + (int)touched.size();
      L1->col.insert(L1->col.end(), touched.begin(), touched.end());
      maxr = std::max(maxr, (int)touched.size());
    }
    L1->nb = (int)L1->col.size();
    L1->maxRowBlocks = maxr;
    L1->diag.assign(na, 0);
    for (int I = 0; I < na; I++)
      for (int k = L1->rowPtr[I]; k < L1->rowPtr[I + 1]; k++)
        if (L1->col[k] == I) { L1->diag[I] = k; break; }
  }
  c.shells.push_back(L1);
  // ---- coarse shell levels (MultigridPC constructor, 10-solver.js:632-644)
  for (int guard = 0; guard < 20; guard++) {
    ShellLevel& cur = *c.shells.back();
    column_factor_sizes(cur);
    const int ncol = cur.nx * cur.ny, ndof = 6 * cur.nn;
    if (ncol <= 9 || ndof <= 900 || (cur.nx <= 2 && cur.ny <= 2)) break;   // MG_COARSEST_COLS, MG_COARSEST_DOF
    const int ncx = (int)coarse_lines(cur.nx, cur.hasKeep ? &cur.keepX : nullptr).size();
    const int ncyy = (int)coarse_lines(cur.ny, cur.hasKeep ? &cur.keepY : nullptr).size();
    if (ncx * ncyy > 0.7 * ncol) break;                                      // MG_MIN_COARSENING
    c.shells.push_back(build_coarse_shell(cur));
  }
  ShellLevel& co = *c.shells.back();
  co.coarsest = true;
  {
    int bw = 0;
    for (int i = 0; i < co.nn; i++)
      for (int k = co.rowPtr[i]; k < co.rowPtr[i + 1]; k++) bw = std::max(bw, std::abs(co.col[k] - i));
    co.bandBw = (bw + 1) * 6 - 1;
    co.denseN = 6 * co.nn;
  }
  // ---- device upload of the structure
  cudaStream_t st = c.stream;
  color_lists(nx, ny, c.colStart, c.d_colorCols, c.colorCount, st);
  // level-0 column panels: greedy packing of each colour's columns (in list order) into groups of
  // at most panelCap nodes; a column longer than panelCap forms a group of its own
  c.panelCap = std::max(TM_PANEL_THREADS, c.maxColLen);
  c.panelMaxCols = 0;
  std::vector<int> colPos[4];
  c.colourPos[0] = 0;
  for (int k = 0; k < 4; k++) {
    std::vector<int> cols;
    for (int col = 0; col < nx * ny; col++) {
      if (c.colStart[col + 1] == c.colStart[col]) continue;
      if (((col / ny) & 1) * 2 + ((col % ny) & 1) == k) cols.push_back(col);
    }
    std::vector<int> gs{0};
    int nodes = 0;
    for (size_t q = 0; q < cols.size(); q++) {
      const int len = c.colStart[cols[q] + 1] - c.colStart[cols[q]];
      if (nodes > 0 && nodes + len > c.panelCap) { gs.push_back((int)q); nodes = 0; }
      nodes += len;
    }
    gs.push_back((int)cols.size());
    if (cols.empty()) gs.assign(1, 0);
    for (size_t g = 0; g + 1 < gs.size(); g++) c.panelMaxCols = std::max(c.panelMaxCols, gs[g + 1] - gs[g]);
    c.grpCount[k] = (int)gs.size() - 1;
    c.d_grpStart[k].upload(gs, st);
    std::vector<int> cp(cols.size() + 1, 0);
    for (size_t q = 0; q < cols.size(); q++) {
      cp[q] = c.pos[c.colStart[cols[q]]];
      cp[q + 1] = cp[q] + c.colStart[cols[q] + 1] - c.colStart[cols[q]];
      if (q > 0 && cp[q] != cp[q - 1] + c.colStart[cols[q - 1] + 1] - c.colStart[cols[q - 1]])
        fail(TM_BAD_INPUT, "colour columns are not contiguous in position order");
    }
    c.d_colPos[k].upload(cp, st);
    colPos[k] = cp;
    c.colourPos[k + 1] = c.colourPos[k] + (cp.empty() ? 0 : cp.back() - cp.front());
  }
  if (c.colourPos[4] != nn) fail(TM_BAD_INPUT, "colours do not cover the positions");
  plan_sweep_tma(c, colPos, st);
  c.d_nodeAgg.upload(c.nodeAgg, st);
  c.d_aggPtr.upload(c.aggPtr, st);
  c.d_aggNodes.upload(c.aggNodes, st);
  galerkin_lists01(c, st);
  for (size_t l = 0; l + 1 < c.shells.size(); l++) galerkin_lists_shell(*c.shells[l], *c.shells[l + 1], st);
  c.d_zp.upload(c.zp, st);
  c.d_W01.alloc(18 * (size_t)nn);
  c.d_F.alloc(18 * (size_t)c.nnp);   // position-ordered, rows to the padded stride (the sweep's bulk copies read whole 4-position groups)
  c.d_F.zero(st);
  c.d_res0.alloc(3 * (size_t)nn);
  for (size_t l = 0; l < c.shells.size(); l++) {
    ShellLevel& L = *c.shells[l];
    L.maxColBlocks = 0;
    for (int cc = 0; cc < L.nx * L.ny; cc++)
      L.maxColBlocks = std::max(L.maxColBlocks, L.rowPtr[L.colStart[cc + 1]] - L.rowPtr[L.colStart[cc]]);
    L.d_rowPtr.upload(L.rowPtr, st);
    L.d_col.upload(L.col, st);
    L.d_val.alloc(36 * (size_t)L.nb);
    L.d_colStart.upload(L.colStart, st);
    L.d_cfPtr.upload(L.cfPtr, st);
    if (!L.coarsest) {
      L.d_cf.alloc((size_t)L.cfPtr.back());
      L.d_cfInv.alloc((size_t)L.cfPtr.back());
    }
    color_lists(L.nx, L.ny, L.colStart, L.d_colorCols, L.colorCount, st);
    shell_column_meta(L, st);
    if (l + 1 < c.shells.size()) {
      L.d_prolPtr.upload(L.prolPtr, st);
      L.d_prolIdx.upload(L.prolIdx, st);
      L.d_prolW.upload(L.prolW, st);
      L.d_chPtr.upload(L.chPtr, st);
      L.d_chIdx.upload(L.chIdx, st);
      L.d_chW.upload(L.chW, st);
    }
    L.d_b.alloc(6 * (size_t)L.nn);
    L.d_x.alloc(6 * (size_t)L.nn);
    L.d_res.alloc(6 * (size_t)L.nn);
    if (L.coarsest) {
      L.d_band.alloc((size_t)L.denseN * (L.bandBw + 1));
      L.d_inv.alloc((size_t)L.denseN * L.denseN);
    }
  }
  c.hierarchy = true;
}

}  // namespace tmg
