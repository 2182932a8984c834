// twins-b200: the RDMA model's slot kernel. One persistent cooperative launch runs many slots: a
// warp owns NIC hosts and switches (the same ones every slot, so their records stay in its SM's L1)
// and runs each one's events of the slot (tr_sim.cuh: host_slot, switch_slot); a grid barrier ends
// the slot and its last block applies the slot's end (finish, exact idle skip). Every wait is
// bounded: a barrier that waits too long sets the run's error flag and the launch returns.
// (reference: rdma_slot / rdma_persist / slot_end, src/rdma/rstep.cuh:3451-3577, 4020-4214)
#include "tr_kernel.h"

namespace tr
{

constexpr long long BARRIER_SPIN_LIMIT = 1ll << 22; // polls of ~64 ns: a quarter of a second or more

__device__ __forceinline__ unsigned ld_volatile(const unsigned *p) { return *(const volatile unsigned *)p; }
#ifdef TR_PROFILE
__device__ __forceinline__ unsigned long long gtimer()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
#endif

// a block's scratch in shared memory: per warp a NIC's DCQCN timers and staged arrivals, or one
// switch's ports, staged arrivals, a safe slot's order and flags
__host__ __device__ inline size_t host_scratch_bytes()
{
    return (sizeof(Due) * MAX_DUE + sizeof(SArr) * HOST_STAGE + sizeof(HPre) * HOST_STAGE + 15) & ~(size_t)15;
}
__host__ __device__ inline size_t sw_ports_bytes(int max_deg) { return ((size_t)max_deg * sizeof(SwPort) + 15) & ~(size_t)15; }
__host__ __device__ inline size_t sw_frames_bytes() { return sizeof(Frame) * SW_FRAMES; }
__host__ __device__ inline size_t block_scratch_bytes(int max_deg)
{
    const size_t host = host_scratch_bytes() * RDMA_WARPS;
    const size_t sw = sw_frames_bytes() + sw_ports_bytes(max_deg) + sizeof(SArr) * SW_STAGE + sizeof(uint16_t) * SW_STAGE + 4 * sizeof(int);
    return ((host > sw ? host : sw) + 15) & ~(size_t)15;
}

// A block's units: a group of RDMA_WARPS NIC hosts (a warp each) or one switch (all its warps: its
// egress ports spread over them in safe slots).
__global__ void __launch_bounds__(RDMA_WARPS * 32) rdma_slot_kernel(RSim s, int slots, int max_deg)
{
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ int blk_last;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    Due *due = reinterpret_cast<Due *>(smem + host_scratch_bytes() * warp);
    SArr *hstage = reinterpret_cast<SArr *>(smem + host_scratch_bytes() * warp + sizeof(Due) * MAX_DUE);
    HPre *hpre = reinterpret_cast<HPre *>(smem + host_scratch_bytes() * warp + sizeof(Due) * MAX_DUE + sizeof(SArr) * HOST_STAGE);
    SwWork work;
    unsigned char *sw = smem;
    work.fr = reinterpret_cast<Frame *>(sw);
    sw += sw_frames_bytes();
    work.port = reinterpret_cast<SwPort *>(sw);
    sw += sw_ports_bytes(max_deg);
    work.arr = reinterpret_cast<SArr *>(sw);
    sw += sizeof(SArr) * SW_STAGE;
    work.ord = reinterpret_cast<uint16_t *>(sw);
    sw += sizeof(uint16_t) * SW_STAGE;
    work.flags = reinterpret_cast<int *>(sw);
    RCtl *ctl = s.ctl;
    volatile RCtl *vc = ctl;
    const int groups = (s.H + RDMA_WARPS - 1) / RDMA_WARPS, units = groups + s.S;
    for (int it = 0; it < slots; it++)
    {
        if (vc->finished)
            return;
        const int64_t t = vc->slot;
        for (int u = blockIdx.x; u < units; u += gridDim.x)
        {
#ifdef TR_PROFILE
            const unsigned long long p0 = gtimer();
#endif
            if (u < groups)
            {
                const int h = u * RDMA_WARPS + warp;
                if (h < s.H)
                {
                    int64_t w = INT64_MAX;
                    const bool act = host_slot(s, h, t, &w, due, hstage, hpre, lane, 32);
                    if (lane == 0)
                    {
                        if (act)
                            atomicAdd(&ctl->activity, 1u);
                        if (w != INT64_MAX)
                            atomicMin(&ctl->next_wake, (unsigned long long)w);
                    }
                }
            }
            else
            {
                if (switch_slot(s, u - groups, t, work, threadIdx.x, RDMA_WARPS * 32) && threadIdx.x == 0)
                    atomicAdd(&ctl->activity, 1u);
            }
#ifdef TR_PROFILE
            if (lane == 0)
                atomicMax(u < groups ? &ctl->prof_host_max : &ctl->prof_sw_max, gtimer() - p0);
#endif
            __syncthreads(); // (the scratch is the next unit's)
        }
        __syncthreads();
        unsigned g = 0;
        if (threadIdx.x == 0)
        {
            g = ld_volatile(&ctl->gen);
            __threadfence();
            blk_last = atomicAdd(&ctl->arrive, 1u) + 1 == gridDim.x;
        }
        __syncthreads();
        if (threadIdx.x == 0)
        {
            if (blk_last)
            {
                __threadfence();
                const unsigned act = atomicExch(&ctl->activity, 0u);
                const unsigned long long wake = atomicExch(&ctl->next_wake, ~0ull);
                const unsigned done = atomicAdd(&ctl->flows_done, 0u);
                slot_close(s, t, act, wake, done);
#ifdef TR_PROFILE
                const unsigned long long now = gtimer();
                if (vc->prof_release)
                    s.ev[EV_PROF_SLOT_NS] += now - vc->prof_release;
                vc->prof_release = now;
                s.ev[EV_PROF_HOST_NS] += atomicExch(&ctl->prof_host_max, 0ull);
                s.ev[EV_PROF_SW_NS] += atomicExch(&ctl->prof_sw_max, 0ull);
                s.ev[EV_PROF_LANE_EV] += atomicExch(&s.ev[EV_PROF_LANE_EV_SLOT], 0ull);
#endif
                vc->arrive = 0;
                __threadfence();
                atomicAdd(&ctl->gen, 1u);
            }
            else
            {
                long long spins = 0;
                while (ld_volatile(&ctl->gen) == g)
                {
                    if (++spins > BARRIER_SPIN_LIMIT)
                    {
                        atomicExch(&ctl->error, 1);
                        atomicExch(&ctl->finished, 1);
                        atomicAdd(&s.ev[EV_TIMEOUT], 1ull);
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

int rdma_launch_shape(int max_deg, int units, int *grid, size_t *smem)
{
    *smem = block_scratch_bytes(max_deg);
    if (cudaFuncSetAttribute((const void *)rdma_slot_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)*smem) != cudaSuccess)
        return (int)cudaGetLastError();
    int dev = 0, sms = 0, per_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, (const void *)rdma_slot_kernel, RDMA_WARPS * 32, *smem) != cudaSuccess)
        return (int)cudaGetLastError();
    if (per_sm < 1)
        return (int)cudaErrorInvalidConfiguration;
    // a block per unit (a group of NIC hosts or a switch) where they fit at once; else every
    // resident block takes several
    *grid = units < per_sm * sms ? units : per_sm * sms;
    return 0;
}

int rdma_launch(const RSim &s, int grid, size_t smem, int slots, int max_deg, cudaStream_t stream)
{
    void *args[] = {(void *)&s, (void *)&slots, (void *)&max_deg};
    const cudaError_t e = cudaLaunchCooperativeKernel((const void *)rdma_slot_kernel, dim3(grid), dim3(RDMA_WARPS * 32), args, smem, stream);
    return e == cudaSuccess ? 0 : (int)e;
}

} // namespace tr
