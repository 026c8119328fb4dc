// Level-0 column smoother of the FP32 V-cycle (columnSweep solid branch + solveColumn,
// src/core/10-solver.js:71-104, 512-534), one colour per launch, as a persistent per-SM sweep:
//
//  * every CTA (one per SM) owns a contiguous run of whole columns of the colour (about 1/148 of
//    the colour's nodes; the colour's positions are contiguous, so the run is one position range);
//  * the run's operator rows (243 values per position) and neighbour ids (27) stream through
//    shared memory in chunks of 64 positions, each chunk one pair of TMA bulk copies
//    (cp.async.bulk, no multicast) of the position-major copies of the operator and the ids (a
//    chunk is one contiguous range of each), completing on an mbarrier, in a ring of stages so
//    that the loads of later chunks are in flight while a chunk's residual rows are computed;
//  * two warp groups take alternate chunks (one group's gathers of x overlap the other's); in a
//    group 4 threads per position take the 27 slots (a warp takes 32 consecutive positions of one
//    slot group, conflict-free), their partial rows are added in a fixed order and the run's
//    residual rows r = b - K x are written to shared memory (b fetched by the chunk itself);
//  * the run's column factors then arrive with one bulk copy into the freed stage memory;
//  * one thread per column then runs the block-tridiagonal forward/backward substitution and
//    the run's x is updated (on the cycle's first sweep, x is assigned and the other colours'
//    nodes are cleared).
//
// Columns of one colour do not couple, so runs never read each other's updates. Every wait on
// an mbarrier is bounded: a wait that runs out sets the error flag, waits (bounded) for the
// copies still in flight and leaves; the host reports TM_TIMEOUT.
#include <cuda_runtime.h>

#include <algorithm>
#include <vector>

#include "tm_internal.h"

namespace tmg {

namespace {

constexpr int TS_THREADS = 512;
constexpr int TS_CHUNK = 64;                                       // positions per chunk (one TMA box)
constexpr int TS_GROUPS = 2;                                       // warp groups, alternate chunks
constexpr int TS_GTHREADS = TS_THREADS / TS_GROUPS;
constexpr int TS_TPP = TS_GTHREADS / TS_CHUNK;                     // threads per position in a group
constexpr int TS_ROWS = NSLOT * 9;                                 // operator rows
constexpr int TS_STAGE_BYTES = (TS_ROWS + NSLOT) * TS_CHUNK * 4;   // values, then neighbour ids
constexpr int TS_MAXSTAGE = 8;
constexpr long long TS_WAIT_LIMIT = 1LL << 22;
constexpr long long TS_TEST_LIMIT = 1LL << 12;                     // the timeout test's wait (see waitTest)
constexpr int TS_ILP = 4;                                          // positions per thread in the run's gathers

__device__ __forceinline__ unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_fence_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, unsigned bytes) {
  asm volatile(
      "{\n"
      " .reg .b64 st;\n"
      " mbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n"
      "}\n" ::"r"(smem_u32(bar)),
      "r"(bytes)
      : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, unsigned parity) {
  unsigned done;
  asm volatile(
      "{\n"
      " .reg .pred p;\n"
      " mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n"
      "}\n"
      : "=r"(done)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return done != 0;
}
// bounded wait for the phase of the given parity
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, unsigned parity) {
  for (long long it = 0; it < TS_WAIT_LIMIT; it++)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
// barrier of one warp group (named barrier 1 + group), and the same with an OR of a flag over
// the group (the same result in every thread of the group)
__device__ __forceinline__ void group_sync(int g) { asm volatile("bar.sync %0, %1;" ::"r"(1 + g), "r"(TS_GTHREADS) : "memory"); }
__device__ __forceinline__ bool group_sync_or(int g, bool v) {
  unsigned r;
  asm volatile(
      "{\n"
      " .reg .pred p, q;\n"
      " setp.ne.u32 p, %1, 0;\n"
      " bar.red.or.pred q, %2, %3, p;\n"
      " selp.u32 %0, 1, 0, q;\n"
      "}\n"
      : "=r"(r)
      : "r"((unsigned)v), "r"(1 + g), "r"(TS_GTHREADS)
      : "memory");
  return r != 0;
}

// L2 policies: the streamed operator rows are read once per sweep (evict first), the gathered
// x is read by every sweep (evict last)
__device__ __forceinline__ uint64_t policy_evict_first() {
  uint64_t p;
  asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
  return p;
}
__device__ __forceinline__ uint64_t policy_evict_last() {
  uint64_t p;
  asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
  return p;
}
__device__ __forceinline__ float ld_keep(const float* p, uint64_t pol) {
  float v;
  asm volatile("ld.global.L2::cache_hint.f32 %0, [%1], %2;" : "=f"(v) : "l"(p), "l"(pol));
  return v;
}

// contiguous bytes into shared memory (16-byte aligned source, destination and size)
__device__ __forceinline__ void bulk_load(void* dst, const void* src, unsigned bytes, uint64_t* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(smem_u32(dst)), "l"(src),
               "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}
// the same with an L2 policy
__device__ __forceinline__ void bulk_load_hint(void* dst, const void* src, unsigned bytes, uint64_t* bar, uint64_t pol) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint [%0], [%1], %2, [%3], %4;" ::"r"(
                   smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(smem_u32(bar)), "l"(pol)
               : "memory");
}

__global__ void __launch_bounds__(TS_THREADS, 1)
    k_sweep_tma(const float* __restrict__ valPm, const int* __restrict__ nbrPm, const int* __restrict__ partCol,
                const int* __restrict__ colPos, const int* __restrict__ posNode, const float* __restrict__ F, const float* __restrict__ b,
                float* __restrict__ x, int maxNodes, int nstage, int zeroGuess, int nn, int zlo, int zhi, int* __restrict__ err,
                int waitTest) {
  extern __shared__ __align__(16) unsigned char smraw_t[];
  __shared__ __align__(8) uint64_t bars[TS_MAXSTAGE + 1];   // chunk stages, then the factors
  // 128-byte aligned start of the stages (the launch adds 128 bytes for this)
  unsigned char* smt = smraw_t + ((128u - (smem_u32(smraw_t) & 127u)) & 127u);
  const int tid = threadIdx.x;
  if (zeroGuess) {
    // the cycle's iterate starts at zero: the nodes of the other colours are cleared here, this
    // colour's are assigned at the end
    const int nOther = nn - (zhi - zlo);
    for (int t = blockIdx.x * blockDim.x + tid; t < nOther; t += gridDim.x * blockDim.x) {
      const size_t n = posNode[t < zlo ? t : t + (zhi - zlo)];
      x[3 * n] = 0; x[3 * n + 1] = 0; x[3 * n + 2] = 0;
    }
  }
  const int c0 = partCol[blockIdx.x], c1 = partCol[blockIdx.x + 1];
  if (c0 >= c1) return;
  const int P0 = colPos[c0], P1 = colPos[c1];
  const int Q0 = P0 & ~3, QE = (P1 + 3) & ~3;   // 16-byte aligned window of the run
  const int nchunks = zeroGuess ? 0 : (QE - Q0 + TS_CHUNK - 1) / TS_CHUNK;
  // the run's factors land in the stage memory once the operator rows have streamed through
  const float* sF = reinterpret_cast<const float*>(smt);                                  // (QE - Q0) x 18
  float* sr = reinterpret_cast<float*>(smt + (size_t)nstage * TS_STAGE_BYTES);            // run rows x 3
  float* red = sr + 3 * (size_t)maxNodes;                                                 // TS_TPP x TS_CHUNK x 3 partial rows
  uint64_t* fbar = &bars[TS_MAXSTAGE];
  if (tid == 0) {
    for (int s = 0; s < nstage; s++) mbar_init(&bars[s], 1);
    mbar_init(fbar, 1);
    mbar_fence_init();
  }
  __syncthreads();
  const uint64_t polStream = policy_evict_first(), polKeep = policy_evict_last();
  __shared__ int s_fail;
  __shared__ int s_last[TS_MAXSTAGE];   // last chunk issued into each stage
  // chunk k: positions Q0 + 64k .. (the last chunk up to QE; both multiples of 4, so every copy
  // starts on a 16-byte boundary and moves a multiple of 16 bytes)
  auto issue = [&](int k) {
    float* dst = reinterpret_cast<float*>(smt + (size_t)(k % nstage) * TS_STAGE_BYTES);
    const int q0 = Q0 + k * TS_CHUNK, np = min(TS_CHUNK, QE - q0);
    const unsigned bv = (unsigned)np * TS_ROWS * 4, bi = (unsigned)np * NSLOT * 4;
    mbar_expect_tx(&bars[k % nstage], bv + bi);
    bulk_load_hint(dst, valPm + (size_t)q0 * TS_ROWS, bv, &bars[k % nstage], polStream);
    bulk_load_hint(dst + TS_ROWS * TS_CHUNK, nbrPm + (size_t)q0 * NSLOT, bi, &bars[k % nstage], polStream);
    s_last[k % nstage] = k;
  };
  if (tid == 0) {
    s_fail = 0;
    for (int q = 0; q < TS_MAXSTAGE; q++) s_last[q] = -1;
    for (int q = 0; q < nstage && q < nchunks; q++) issue(q);
  }
  // r = b - K x: each chunk loads its positions' b while it waits for its stage and computes, and
  // writes r once. On the cycle's first sweep (x = 0, no chunks) r = b, loaded here: a thread
  // takes up to TS_ILP positions and issues their loads together (the node ids, then b)
  const int nrun = P1 - P0;
  for (int l0 = tid; zeroGuess && l0 < nrun; l0 += TS_ILP * blockDim.x) {
    size_t nd[TS_ILP];
    float v[TS_ILP][3];
#pragma unroll
    for (int u = 0; u < TS_ILP; u++) {
      const int l = l0 + u * blockDim.x;
      nd[u] = l < nrun ? (size_t)posNode[P0 + l] : 0;
    }
#pragma unroll
    for (int u = 0; u < TS_ILP; u++)
      if (l0 + u * (int)blockDim.x < nrun) {
        v[u][0] = b[3 * nd[u]]; v[u][1] = b[3 * nd[u] + 1]; v[u][2] = b[3 * nd[u] + 2];
      }
#pragma unroll
    for (int u = 0; u < TS_ILP; u++) {
      const int l = l0 + u * blockDim.x;
      if (l < nrun) { sr[3 * l] = v[u][0]; sr[3 * l + 1] = v[u][1]; sr[3 * l + 2] = v[u][2]; }
    }
  }
  __syncthreads();
  // two warp groups take alternate chunks, so that one group's gathers of x overlap the other's;
  // a warp takes 32 consecutive positions of one slot group: position rows are 243 values and 27
  // ids long (odd strides), so the warp's shared-memory accesses fall in 32 different banks
  const int grp = tid / TS_GTHREADS, gtid = tid % TS_GTHREADS;
  const int pl = gtid % TS_CHUNK, sub = gtid / TS_CHUNK;
  float* gred = red + (size_t)grp * TS_TPP * TS_CHUNK * 3;
  for (int k = grp; k < nchunks; k += TS_GROUPS) {
    // b of the position and component this thread adds the partial rows of (see below)
    const int rq = gtid / 3, rc = gtid % 3, rp = Q0 + k * TS_CHUNK + rq;
    const bool rlive = gtid < 3 * TS_CHUNK && rp >= P0 && rp < P1;
    const float bv = rlive ? b[3 * (size_t)posNode[rp] + rc] : 0.f;
    // the chunk's loads must have been issued before its stage is waited on: the previous chunk
    // of the stage belongs to the other group, and a wait one phase early would see that phase
    // (waitTest: the test hook of the timeout path waits, with a short limit, for a stage number that
    // is never issued)
    bool ok = false;
    const int want = waitTest ? -2 : k;
    const long long limit = waitTest ? TS_TEST_LIMIT : TS_WAIT_LIMIT;
    for (long long it = 0; it < limit; it++)
      if (*(volatile int*)&s_last[k % nstage] == want) { ok = true; break; }
    if (ok) ok = mbar_wait(&bars[k % nstage], (unsigned)(k / nstage) & 1u);
    if (!ok) s_fail = 1;
    const float* sv = reinterpret_cast<const float*>(smt + (size_t)(k % nstage) * TS_STAGE_BYTES);
    const int* sn = reinterpret_cast<const int*>(sv + TS_ROWS * TS_CHUNK);
    const int p = Q0 + k * TS_CHUNK + pl;
    const bool live = ok && p >= P0 && p < P1;
    float a0 = 0, a1 = 0, a2 = 0;
    if (live) {
#pragma unroll
      for (int h = 0; h < (NSLOT + TS_TPP - 1) / TS_TPP; h++) {
        const int s = sub + TS_TPP * h;
        if (s < NSLOT) {
          const int jj = sn[pl * NSLOT + s];
          const size_t j = jj < 0 ? 0 : jj;   // absent slots hold zeros
          const float x0 = ld_keep(x + 3 * j, polKeep), x1 = ld_keep(x + 3 * j + 1, polKeep), x2 = ld_keep(x + 3 * j + 2, polKeep);
          const float* v = sv + pl * TS_ROWS + s * 9;
          a0 += v[0] * x0 + v[1] * x1 + v[2] * x2;
          a1 += v[3] * x0 + v[4] * x1 + v[5] * x2;
          a2 += v[6] * x0 + v[7] * x1 + v[8] * x2;
        }
      }
    }
    float* rd = gred + 3 * (size_t)(sub * TS_CHUNK + pl);
    rd[0] = a0; rd[1] = a1; rd[2] = a2;
    // the stage is read: refill it while the partial rows are added (every thread of the group
    // takes the same branch)
    if (group_sync_or(grp, !ok || *(volatile int*)&s_fail != 0)) {
      s_fail = 1;
      break;
    }
    if (gtid == 0 && k + nstage < nchunks) {
      fence_proxy_async();   // the stage being refilled was last read by the threads
      issue(k + nstage);
    }
    // the slot groups' partial rows of a position, added in group order: r = b - (K x)
    if (rlive) {
      float acc = gred[3 * rq + rc];
#pragma unroll
      for (int g = 1; g < TS_TPP; g++) acc += gred[3 * (g * TS_CHUNK + rq) + rc];
      sr[3 * (rp - P0) + rc] = bv - acc;
    }
    group_sync(grp);
  }
  __syncthreads();
  bool failed = s_fail != 0;
  bool fIssued = false;   // thread 0
  if (!failed && tid == 0) {
    // the factors into the (now free) stage memory
    const unsigned fbytes = (unsigned)(QE - Q0) * 18 * 4;
    fence_proxy_async();
    mbar_expect_tx(fbar, fbytes);
    bulk_load(smt, F + 18 * (size_t)Q0, fbytes, fbar);
    fIssued = true;
  }
  if (!failed) {
    const bool ok = mbar_wait(fbar, 0);
    failed = __syncthreads_or(!ok) != 0;
  }
  if (failed) {
    // give up: flag it, let the copies still in flight land (bounded), leave
    if (tid == 0) {
      atomicExch(err, 1);
      for (int q = 0; q < nstage; q++)
        if (s_last[q] >= 0) mbar_wait(&bars[q], (unsigned)(s_last[q] / nstage) & 1u);
      if (fIssued) mbar_wait(fbar, 0);
    }
    __syncthreads();
    return;
  }
  // one thread per column: block-tridiagonal forward and backward substitution (scalar loads: a
  // float2 version of the factor reads measured slower, 6.3 against 4.9 µs per launch, as the
  // 8-byte accesses of neighbouring columns conflict in more banks)
  for (int q = tid; q < c1 - c0; q += blockDim.x) {
    const int cp0 = colPos[c0 + q], len = colPos[c0 + q + 1] - cp0;
    float* rr = sr + 3 * (size_t)(cp0 - P0);
    const float* Fc = sF + 18 * (size_t)(cp0 - Q0);
    float p0v = 0, p1v = 0, p2v = 0;
    for (int l = 0; l < len; l++) {
      const float* f = Fc + 18 * l;
      float b0 = rr[3 * l], b1 = rr[3 * l + 1], b2 = rr[3 * l + 2];
      if (l > 0) {
        b0 -= f[9] * p0v + f[10] * p1v + f[11] * p2v;
        b1 -= f[12] * p0v + f[13] * p1v + f[14] * p2v;
        b2 -= f[15] * p0v + f[16] * p1v + f[17] * p2v;
      }
      const float y0 = b0 * f[1];
      const float y1 = (b1 - f[3] * y0) * f[2];
      const float y2 = (b2 - f[6] * y0 - f[7] * y1) * f[5];
      rr[3 * l] = y0; rr[3 * l + 1] = y1; rr[3 * l + 2] = y2;
      p0v = y0; p1v = y1; p2v = y2;
    }
    float q0 = 0, q1 = 0, q2 = 0;
    for (int l = len - 1; l >= 0; l--) {
      const float* f = Fc + 18 * l;
      float b0 = rr[3 * l], b1 = rr[3 * l + 1], b2 = rr[3 * l + 2];
      if (l + 1 < len) {
        const float* g = Fc + 18 * (l + 1);
        b0 -= g[9] * q0 + g[12] * q1 + g[15] * q2;
        b1 -= g[10] * q0 + g[13] * q1 + g[16] * q2;
        b2 -= g[11] * q0 + g[14] * q1 + g[17] * q2;
      }
      const float z2 = b2 * f[5];
      const float z1 = (b1 - f[7] * z2) * f[2];
      const float z0 = (b0 - f[3] * z1 - f[6] * z2) * f[1];
      rr[3 * l] = z0; rr[3 * l + 1] = z1; rr[3 * l + 2] = z2;
      q0 = z0; q1 = z1; q2 = z2;
    }
  }
  __syncthreads();
  // x of the run (node ids, then x, then the stores, TS_ILP positions per thread)
  for (int l0 = tid; l0 < nrun; l0 += TS_ILP * blockDim.x) {
    size_t nd[TS_ILP];
#pragma unroll
    for (int u = 0; u < TS_ILP; u++) {
      const int l = l0 + u * blockDim.x;
      nd[u] = l < nrun ? (size_t)posNode[P0 + l] : 0;
    }
    if (zeroGuess) {
#pragma unroll
      for (int u = 0; u < TS_ILP; u++) {
        const int l = l0 + u * blockDim.x;
        if (l < nrun) { x[3 * nd[u]] = sr[3 * l]; x[3 * nd[u] + 1] = sr[3 * l + 1]; x[3 * nd[u] + 2] = sr[3 * l + 2]; }
      }
    } else {
      float v[TS_ILP][3];
#pragma unroll
      for (int u = 0; u < TS_ILP; u++)
        if (l0 + u * (int)blockDim.x < nrun) {
          v[u][0] = x[3 * nd[u]]; v[u][1] = x[3 * nd[u] + 1]; v[u][2] = x[3 * nd[u] + 2];
        }
#pragma unroll
      for (int u = 0; u < TS_ILP; u++) {
        const int l = l0 + u * blockDim.x;
        if (l < nrun) {
          x[3 * nd[u]] = v[u][0] + sr[3 * l]; x[3 * nd[u] + 1] = v[u][1] + sr[3 * l + 1]; x[3 * nd[u] + 2] = v[u][2] + sr[3 * l + 2];
        }
      }
    }
  }
}

}  // namespace

inline int grid_for(size_t n, int block) { return (int)((n + block - 1) / block); }

// FP32 copies of the level-0 operator in one pass over the FP64 one: slot-major (rows of nnp
// positions, as the FP64 operator; the apply and the panel sweep read it) and, when vpm is
// given, position-major (the 243 values of a position contiguous, the layout the TMA sweep
// streams). A block takes 32 positions: coalesced row reads, a shared-memory transpose, one
// contiguous write.
__global__ void __launch_bounds__(256) k_val_to_f32(int nnp, const double* __restrict__ val, float* __restrict__ v32,
                                                    float* __restrict__ vpm) {
  __shared__ float tile[32 * TS_ROWS];
  const int p0 = blockIdx.x * 32, pl = threadIdx.x & 31, p = p0 + pl;
  for (int r = threadIdx.x >> 5; r < TS_ROWS; r += 8) {
    float f = 0.f;
    if (p < nnp) {
      f = (float)val[(size_t)r * nnp + p];
      v32[(size_t)r * nnp + p] = f;
    }
    tile[pl * TS_ROWS + r] = f;   // bank (19 pl + r) mod 32: conflict-free
  }
  if (!vpm) return;
  __syncthreads();
  const int np = min(32, nnp - p0);
  float* out = vpm + (size_t)p0 * TS_ROWS;
  for (int j = threadIdx.x; j < np * TS_ROWS; j += blockDim.x) out[j] = tile[j];
}

// position-major copy of the neighbour ids (27 per position)
__global__ void k_nbr_pm(int nnp, const int* __restrict__ nbr, int* __restrict__ npm) {
  const size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (t >= (size_t)nnp * NSLOT) return;
  const int p = (int)(t / NSLOT), s = (int)(t % NSLOT);
  npm[t] = nbr[(size_t)s * nnp + p];
}

// shared memory of the sweep for the longest run; 0 when even two stages do not fit
size_t sweep_tma_smem(int maxNodes, int nstage) {
  if ((size_t)(maxNodes + 8) * 18 * 4 > (size_t)nstage * TS_STAGE_BYTES) return ~(size_t)0;   // the factors reuse the stages
  return 128 + (size_t)nstage * TS_STAGE_BYTES + (size_t)maxNodes * 3 * 4 + (size_t)TS_THREADS * 3 * 4;
}

// runs of whole columns per colour, one per SM, with about equal node counts; the number of
// chunk stages that fits beside the longest run's factors and rows (0: the sweep is not used)
void plan_sweep_tma(Context& c, const std::vector<int>* colPos, cudaStream_t st) {
  int sms = 0, smemMax = 0;
  TM_CUDA_CHECK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c.dev));
  TM_CUDA_CHECK(cudaDeviceGetAttribute(&smemMax, cudaDevAttrMaxSharedMemoryPerBlockOptin, c.dev));
  c.tsParts = std::max(1, sms);
  c.tsMaxNodes = 0;
  std::vector<int> parts[4];
  for (int k = 0; k < 4; k++) {
    const std::vector<int>& cp = colPos[k];
    const int ncols = (int)cp.size() - 1;
    const long long total = ncols > 0 ? cp[ncols] - cp[0] : 0;
    std::vector<int>& part = parts[k];
    part.assign(c.tsParts + 1, 0);
    int q = 0;
    for (int p = 0; p < c.tsParts; p++) {
      part[p] = q;
      const long long target = total * (p + 1) / c.tsParts;
      while (q < ncols && cp[q + 1] - cp[0] <= target) q++;
    }
    part[c.tsParts] = std::max(ncols, 0);
    for (int p = 0; p < c.tsParts; p++) c.tsMaxNodes = std::max(c.tsMaxNodes, cp[part[p + 1]] - cp[part[p]]);
    c.d_tsPart[k].upload(part, st);
  }
  const size_t staticSmem = 256;   // the kernel's barriers and flags
  c.tsStages = 0;
  for (int ns = 3; ns >= 2 && !c.tsStages; ns--) {
    const size_t need = sweep_tma_smem(c.tsMaxNodes, ns);   // ~0 (does not fit) must not wrap when the static part is added
    if (need != ~(size_t)0 && need + staticSmem <= (size_t)smemMax) c.tsStages = ns;
  }
  c.tsPlanned = c.tsStages;
  c.tsReady = TM_SWEEP_TMA && c.tsStages > 0;
  if (c.tsReady) {
    c.d_nbrp.alloc((size_t)NSLOT * c.nnp);
    k_nbr_pm<<<grid_for((size_t)NSLOT * c.nnp, 256), 256, 0, st>>>(c.nnp, c.d_nbr.p, c.d_nbrp.p);
    note_launch();
    TM_CUDA_CHECK(cudaGetLastError());
  }
}

bool launch_sweep_tma(Context& c, int col, int zeroGuess, const float* b, float* x) {
  if (!c.tsReady) return false;
  const size_t smem = sweep_tma_smem(c.tsMaxNodes, c.tsStages);
  TM_CUDA_CHECK(cudaFuncSetAttribute(k_sweep_tma, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  k_sweep_tma<<<c.tsParts, TS_THREADS, smem, c.stream>>>(c.d_val32p.p, c.d_nbrp.p, c.d_tsPart[col].p, c.d_colPos[col].p, c.d_posNode.p,
                                                        c.d_F32.p, b, x, c.tsMaxNodes, c.tsStages, zeroGuess, c.nn, c.colourPos[col],
                                                        c.colourPos[col + 1], c.d_err.p, c.waitTest ? 1 : 0);
  note_launch();
  return true;
}

void launch_val_to_f32(Context& c) {
  const size_t n = (size_t)TS_ROWS * c.nnp;
  c.d_val32.alloc(n);
  if (c.tsReady) c.d_val32p.alloc(n);
  k_val_to_f32<<<(c.nnp + 31) / 32, 256, 0, c.stream>>>(c.nnp, c.d_val.p, c.d_val32.p, c.tsReady ? c.d_val32p.p : nullptr);
  note_launch();
  TM_CUDA_CHECK(cudaGetLastError());
}

}  // namespace tmg
