// twins-b200: launching the slot kernel (host side).
#pragma once
#include <cuda_runtime.h>

#ifndef TB_WARPS_PER_BLOCK
#define TB_WARPS_PER_BLOCK 4
#endif

namespace tb
{
struct Sim;
// blocks of the slot kernel that fit on one SM at once (0 on error)
int slot_kernel_blocks_per_sm(int stage_cap, bool port_local = false, int host_lanes = 1);
// one cooperative launch of up to max_slots_per_launch slots; 0 or a cudaError_t
// port_local: switch ports keep the slot's transmission chain and last enqueued frame in shared memory
int launch_slots(const Sim &s, int grid, int max_slots_per_launch, int host_lanes, int stage_cap, bool port_local, cudaStream_t stream);
// a cached graph of one launch (launch_slots_graph)
struct SlotGraph
{
    void *exec = nullptr;
    unsigned long long key[8] = {};
    bool broken = false;      // capture failed: plain launches
    long long replays = 0;
};
// launch_slots through a CUDA graph, captured once per shape, slot count and unit list
int launch_slots_graph(SlotGraph &g, const Sim &s, int grid, int max_slots_per_launch, int host_lanes, int stage_cap, bool port_local,
                       cudaStream_t stream);
void release_graph(SlotGraph &g);
} // namespace tb
