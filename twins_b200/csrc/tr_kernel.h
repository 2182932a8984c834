// twins-b200: the RDMA slot kernel's launch (tr_kernel.cu), for the C ABI.
#pragma once
#include "tr_sim.cuh"

#include <cuda_runtime.h>

namespace tr
{

constexpr int RDMA_WARPS = 4; // warps per block

// the cooperative launch's grid and dynamic shared memory for switches of at most max_deg ports;
// units: groups of RDMA_WARPS NIC hosts plus switches; 0 or a CUDA error
int rdma_launch_shape(int max_deg, int units, int *grid, size_t *smem);
// up to `slots` slots of the run s (stops early when it finishes); 0 or a CUDA error
int rdma_launch(const RSim &s, int grid, size_t smem, int slots, int max_deg, cudaStream_t stream);

} // namespace tr
