// twins-b200: the persistent slot kernel.
//
// One cooperative launch runs up to `max_slots_per_launch` slots of every world in the batch.
// Warps own entities for the whole launch (host units of `host_lanes` hosts, one thread each;
// one switch per warp, one lane per port), so each entity's records stay in its SM's L1; link
// messages cross SMs through L2 (ld/st.cg). Slots are separated by a grid barrier whose last
// arriving block does the slot bookkeeping of the reference's ticket block
// (src/kernel.cuh:79-112): finish when every message is done, else the exact idle skip to the
// earliest host wake-up when nothing was sent in this or the previous slot. Every wait is
// bounded; a barrier that times out sets an error flag and ends the launch.
#include "tb_switch.cuh"
#include "tb_kernel.h"

#include <cuda_runtime.h>

namespace tb
{

constexpr int WARPS_PER_BLOCK = TB_WARPS_PER_BLOCK;
constexpr long long BARRIER_SPIN_LIMIT = 1ll << 22; // polls of >= 64 ns: several seconds

__device__ __forceinline__ unsigned ld_acquire(const unsigned *p)
{
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// one switch, one slot, by its warp (lanes >= k idle but take part in the warp barriers)
__device__ bool switch_step(const Sim &s, int sw, int64_t t, int lane, SwShared &sh, unsigned &ties)
{
    const SwRec &sr = s.sws[sw];
    SwCtx x;
    x.s = &s;
    x.wd = &s.worlds[sr.world];
    x.sr = &sr;
    x.sw = sw;
    x.ports = s.ports + sr.port0;
    x.scratch = (size_t)sw * s.kmax * 2 * MAX_TX;
    x.t = t;
    x.spray = x.wd->spray != 0;
    const int k = sr.k;
    const bool on = lane < k;
    unsigned pk = 0, drops = 0, marks = 0, ovf = 0, my_ties = 0;
    if (on)
        pk = sw_phase_window(x, sh, lane);
    __syncwarp();
    if (x.spray)
    {
        if (lane == 0)
            sw_phase_spray(x, sh, my_ties);
        __syncwarp();
    }
    if (on)
        drops += sw_phase_count(x, sh, lane);
    __syncwarp();
    if (on)
        sw_phase_offsets(x, sh, lane);
    __syncwarp();
    if (on)
        sw_phase_base(x, sh, lane);
    __syncwarp();
    if (on)
        sw_phase_scatter(x, sh, lane);
    __syncwarp();
    bool act = false;
    if (on)
        act = sw_phase_egress(x, sh, lane, my_ties, drops, marks, ovf);
    // warp totals, one atomic each
    for (int o = 16; o > 0; o >>= 1)
    {
        pk += __shfl_xor_sync(0xffffffffu, pk, o);
        drops += __shfl_xor_sync(0xffffffffu, drops, o);
        marks += __shfl_xor_sync(0xffffffffu, marks, o);
        ovf += __shfl_xor_sync(0xffffffffu, ovf, o);
        my_ties += __shfl_xor_sync(0xffffffffu, my_ties, o);
    }
    bool any = __any_sync(0xffffffffu, act);
    if (lane == 0)
    {
        ev_add(s, sr.world, EV_SW_PKT, pk);
        ev_add(s, sr.world, EV_DROPS, drops);
        ev_add(s, sr.world, EV_MARKS, marks);
        ev_add(s, sr.world, EV_OVF_TX, ovf);
        ev_add(s, sr.world, EV_TIES, my_ties);
        ties += my_ties;
    }
    return any;
}

__global__ void __launch_bounds__(WARPS_PER_BLOCK * 32) slot_kernel(Sim s, int max_slots_per_launch, int host_lanes)
{
    __shared__ SwShared sw_sh[WARPS_PER_BLOCK];
    __shared__ unsigned blk_act, blk_done;
    __shared__ unsigned long long blk_wake;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int gwarp = blockIdx.x * WARPS_PER_BLOCK + warp, nwarps = gridDim.x * WARPS_PER_BLOCK;
    const int host_units = (s.H + host_lanes - 1) / host_lanes;
    const int units = host_units + s.S;
    SlotCtl *ctl = s.ctl;
    for (int it = 0; it < max_slots_per_launch; it++)
    {
        if (threadIdx.x == 0)
        {
            blk_act = 0;
            blk_done = 0;
            blk_wake = ~0ull;
        }
        __syncthreads();
        // (written by the last block of the previous barrier, before it released the others)
        if (*(volatile int *)&ctl->finished)
            return;
        const int64_t t = *(volatile int64_t *)&ctl->slot;
        unsigned ties = 0;
        for (int u = gwarp; u < units; u += nwarps)
        {
            if (u < host_units)
            {
                int h = u * host_lanes + lane;
                if (lane < host_lanes && h < s.H)
                {
                    int64_t w = INT64_MAX;
                    unsigned done = 0;
                    if (host_step(s, h, t, &w, &ties, &done))
                        atomicOr(&blk_act, 1u);
                    if (done)
                        atomicAdd(&blk_done, done);
                    atomicMin(&blk_wake, (unsigned long long)w);
                }
            }
            else if (switch_step(s, u - host_units, t, lane, sw_sh[warp], ties) && lane == 0)
                atomicOr(&blk_act, 1u);
        }
        __syncthreads();
        if (threadIdx.x == 0)
        {
            if (blk_act)
                atomicOr(&ctl->act_cur, 1u);
            if (blk_wake != ~0ull)
                atomicMin(&ctl->next_wake, blk_wake);
            if (blk_done)
                atomicAdd(&ctl->flows_done, blk_done);
            // grid barrier: the last block to arrive ends the slot and releases the others
            unsigned g = ld_acquire(&ctl->gen);
            __threadfence();
            unsigned arrived = atomicAdd(&ctl->arrive, 1u) + 1;
            if (arrived == gridDim.x)
            {
                __threadfence();
                ctl->arrive = 0;
                unsigned fd = atomicAdd(&ctl->flows_done, 0u);
                if (fd >= (unsigned)s.M || t + 1 >= s.max_slots)
                    ctl->finished = 1;
                unsigned cur = atomicAdd(&ctl->act_cur, 0u), prev = ctl->act_prev;
                unsigned long long nw = atomicAdd(&ctl->next_wake, 0ull);
                int64_t next = t + 1;
                if (cur == 0 && prev == 0 && nw != ~0ull && (int64_t)nw > next)
                    next = (int64_t)nw < s.max_slots ? (int64_t)nw : s.max_slots;
                ctl->act_prev = cur;
                ctl->act_cur = 0;
                ctl->next_wake = ~0ull;
                ctl->slot = next;
                ctl->slots_run++;
                __threadfence();
                atomicAdd(&ctl->gen, 1u);
            }
            else
            {
                long long spins = 0;
                while (ld_acquire(&ctl->gen) == g)
                {
                    if (++spins > BARRIER_SPIN_LIMIT)
                    {
                        atomicExch(&ctl->error, 1);
                        atomicExch(&ctl->finished, 1);
                        atomicAdd(&s.ev[EV_BARRIER_TIMEOUT], 1ull);
                        break;
                    }
                    __nanosleep(64);
                }
            }
            __threadfence();
        }
        __syncthreads();
    }
}

int slot_kernel_blocks_per_sm()
{
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, slot_kernel, WARPS_PER_BLOCK * 32, 0) != cudaSuccess)
        return 0;
    return n;
}

int launch_slots(const Sim &s, int grid, int max_slots_per_launch, int host_lanes, cudaStream_t stream)
{
    void *args[] = {(void *)&s, (void *)&max_slots_per_launch, (void *)&host_lanes};
    cudaError_t e = cudaLaunchCooperativeKernel((const void *)slot_kernel, dim3(grid), dim3(WARPS_PER_BLOCK * 32), args, 0, stream);
    return e == cudaSuccess ? 0 : (int)e;
}

} // namespace tb
