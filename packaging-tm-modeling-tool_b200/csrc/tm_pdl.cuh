// Programmatic dependent launch of the V-cycle's kernels.
//
// A grid launched by launch_pdl may start while the previous kernel of the stream drains: it
// first reads only data that no kernel of the V-cycle writes (operator blocks and rows, ids,
// column factors and inverses, run tables), then waits in grid_dep_wait until every earlier kernel
// has completed and its writes are visible (a no-op in a grid launched without the attribute).
// grid_dep_launch lets the next such grid start once every CTA of this one has issued it.
//
// The wait does not clear the SM's L1, which CTAs of the earlier grids running on the same SM may
// have filled with lines that other SMs wrote since: what earlier kernels write (iterates,
// right-hand sides, residuals) is read after the wait with ld.global.cg (L2, the point of
// coherence).
#pragma once
#include <cuda_runtime.h>

#include "tm_internal.h"

namespace tmg {

__device__ __forceinline__ void grid_dep_wait() { asm volatile("griddepcontrol.wait;\n" ::: "memory"); }
__device__ __forceinline__ void grid_dep_launch() { asm volatile("griddepcontrol.launch_dependents;\n" ::: "memory"); }

template <class... KArgs, class... Args>
inline void launch_pdl(void (*kern)(KArgs...), int grid, int block, size_t smem, cudaStream_t st, Args... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)grid);
  cfg.blockDim = dim3((unsigned)block);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  TM_CUDA_CHECK(cudaLaunchKernelEx(&cfg, kern, args...));
}

}  // namespace tmg
