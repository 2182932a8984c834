// twins-b200: launching the slot kernel (host side).
#pragma once
#include <cuda_runtime.h>

#ifndef TB_WARPS_PER_BLOCK
#define TB_WARPS_PER_BLOCK 4
#endif

namespace tb
{
struct Sim;
// blocks of the slot kernel (free: the batch kernel without a grid barrier) that fit on one SM at
// once (0 on error)
int slot_kernel_blocks_per_sm(int stage_cap, bool port_local = false, int host_lanes = 1, bool free = false);
// one cooperative launch of up to max_slots_per_launch slots; 0 or a cudaError_t
// port_local: switch ports keep the slot's transmission chain and last enqueued frame in shared memory
int launch_slots(const Sim &s, int grid, int max_slots_per_launch, int host_lanes, int stage_cap, bool port_local, cudaStream_t stream);
// A batch launch without a grid barrier: every world runs up to slots_per_world slots on a barrier
// of its own, over the unit list s.unit_list (host units: first host h < H, hosts of one world;
// switches: H + switch) with s.w_units[w] units of world w; s.unit_done holds n_list entries.
// 0 or a cudaError_t
int launch_free(const Sim &s, int grid, int slots_per_world, int host_lanes, int stage_cap, bool port_local, cudaStream_t stream);
// a cached graph of one launch (launch_slots_graph)
struct SlotGraph
{
    void *exec = nullptr;
    unsigned long long key[9] = {};
    bool broken = false;      // capture failed: plain launches
    long long replays = 0;
};
// launch_slots through a CUDA graph, captured once per shape, slot count and unit list
int launch_slots_graph(SlotGraph &g, const Sim &s, int grid, int max_slots_per_launch, int host_lanes, int stage_cap, bool port_local,
                       cudaStream_t stream, bool free = false);
void release_graph(SlotGraph &g);
} // namespace tb
