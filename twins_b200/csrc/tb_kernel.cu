// twins-b200: the persistent slot kernel.
//
// One cooperative launch runs up to `max_slots_per_launch` slots of every world in the batch.
// Warps own entities for the whole launch (host units of `host_lanes` hosts, one thread each;
// one switch per warp, one lane per port), so each entity's records stay in its SM's L1; link
// messages cross SMs through L2 (ld/st.cg). A warp stages the link messages its unit reads in
// shared memory first. Slots are separated by a grid barrier whose last arriving block does the
// slot bookkeeping of the reference's ticket block (src/kernel.cuh:79-112): finish when every
// message is done, else the exact idle skip to the earliest host wake-up when nothing was sent in
// this or the previous slot. Every wait is bounded; a barrier that times out sets an error flag
// and ends the launch.
#include "tb_switch.cuh"
#include "tb_kernel.h"

#include <climits>
#include <cuda_runtime.h>

namespace tb
{

constexpr int WARPS_PER_BLOCK = TB_WARPS_PER_BLOCK;
constexpr long long BARRIER_SPIN_LIMIT = 1ll << 22; // polls of >= 64 ns: several seconds

__device__ __forceinline__ unsigned long long globaltimer()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// The barrier's generation word. Cross-SM data (link messages, the controller) is read from L2
// (ld.cg, volatile, atomics) and every entity's private state stays on its SM, so the wait needs
// no acquire load, which would invalidate the L1 that holds the entities' records.
__device__ __forceinline__ unsigned ld_gen(const unsigned *p)
{
    unsigned v;
    asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void prefetch_l1(const void *p) { asm volatile("prefetch.global.L1 [%0];" ::"l"(p)); }

// Per-packet spraying's draws with staged frames: the merged arrival order by a warp-wide argmin.
// Lane q holds port q's next frame; the minimum (time, longer first) wins; frames that tie on
// both are ordered by lane 0 exactly as the serial merge (sw_phase_spray) orders them, scanning
// the tied ports in port order. Lane 0 keeps the switch's random stream and draws.
__device__ void sw_phase_spray_warp(const SwCtx &x, const SwShared &sh, int lane, unsigned &ties)
{
    const unsigned FULL = 0xffffffffu;
    const int k = x.sr->k;
    const WorldDesc &wd = *x.wd;
    Input in{};
    int cnt = 0, pos = 0;
    if (lane < k)
    {
        in = input_of(x, sh, lane);
        cnt = in.count();
    }
    Rng st;
    if (lane == 0)
        st = x.s->sw_rng[x.sw];
    for (;;)
    {
        const bool has = lane < k && pos < cnt;
        long long kts = has ? in.at(pos)->ts : LLONG_MAX;
        int klen = has ? in.at(pos)->len : 0;
        long long mts = kts;
        int mlen = klen;
        for (int o = 16; o > 0; o >>= 1)
        {
            long long ots = __shfl_xor_sync(FULL, mts, o);
            int olen = __shfl_xor_sync(FULL, mlen, o);
            if (ots < mts || (ots == mts && olen > mlen))
            {
                mts = ots;
                mlen = olen;
            }
        }
        if (mts == LLONG_MAX)
            break;
        const unsigned cand = __ballot_sync(FULL, has && kts == mts && klen == mlen);
        int best = __ffs(cand) - 1;
        if (cand & (cand - 1))
        {
            // equal times and lengths: the upstream chains, then the connection id
            const Frame *bf = nullptr;
            for (unsigned c = cand; c; c &= c - 1)
            {
                int q = __ffs(c) - 1;
                int pq = __shfl_sync(FULL, pos, q);
                if (lane == 0)
                {
                    const Frame *f = input_of(x, sh, q).at(pq);
                    if (!bf || frame_before(*f, *bf, ties))
                    {
                        best = q;
                        bf = f;
                    }
                }
            }
            best = __shfl_sync(FULL, best, 0);
        }
        const int pb = __shfl_sync(FULL, pos, best);
        if (lane == 0)
        {
            const Frame &w = *input_of(x, sh, best).at(pb);
            int ep = wd.n_fail ? epoch_of(wd, w.ts) : 0;
            if (!port_down(wd, x.sr->local, best, ep))
            {
                int nr = routes_to(wd, x.sr->local, w.dst, ep);
                x.s->sw_up[x.scratch + (size_t)best * 2 * MAX_TX + pb] = (uint8_t)(nr ? rand_int(st, (uint32_t)nr) : 0);
            }
        }
        if (lane == best)
            pos++;
    }
    if (lane == 0)
        x.s->sw_rng[x.sw] = st;
}

// A host unit with one host per warp: the warp copies the host's incoming link messages to shared
// memory (one cooperative pass) and prefetches into L1 what the host's events will read: the
// records of the frames' connections with the heads of their sent lists and RTT histories, the
// head frames of the host's egress queue, and the timers of its active connections. Lane 0 then
// runs the host's slot (host_step) on the staged frames. Returns the staging area, or null when
// the messages do not fit it (host_step then reads them in place).
__device__ const Frame *host_prepare(const Sim &s, int h, int64_t t, int lane, SwShared &sh)
{
    const HostRec &hr = s.hosts[h];
    const int link = hr.in_link;
    const int n2 = t >= 2 ? msg_count(s, t - 2, link) : 0, n1 = t >= 1 ? msg_count(s, t - 1, link) : 0, n = n2 + n1;
    if (n == 0 && t < hr.wake && hr.q_size == 0)
        return nullptr; // (nothing to do this slot: host_step returns at once)
    const bool staged = n <= SW_STAGE;
    if (staged)
        for (int i = lane; i < n; i += 32)
            frame_load_link(sh.fr[i], i < n2 ? msg_frames(s, t - 2, link) + i : msg_frames(s, t - 1, link) + (i - n2));
    __syncwarp();
    if (staged)
        for (int i = lane; i < n; i += 32)
        {
            const Frame &f = sh.fr[i];
            if (f.to_sender)
            {
                const SndRec *S = &s.snd[f.flow];
                for (int b = 0; b < (int)sizeof(SndRec); b += 128)
                    prefetch_l1((const char *)S + b);
                const uint64_t off = S->it_off;
                prefetch_l1(&s.it_start[off + S->it_head]);
                prefetch_l1(&s.it_fl[off + S->it_head]);
                const uint32_t hh = S->h_head;
                prefetch_l1(&s.h_seq[off + hh]);
                prefetch_l1(&s.h_cnt[off + hh]);
                prefetch_l1(&s.h_t[off + hh]);
            }
            else
            {
                const RcvRec *R = &s.rcv[f.flow];
                for (int b = 0; b < (int)sizeof(RcvRec); b += 128)
                    prefetch_l1((const char *)R + b);
            }
        }
    if (lane < 8 && lane < hr.q_size)
    {
        int at = hr.q_head + lane;
        if (at >= s.ring)
            at -= s.ring;
        prefetch_l1(&s.host_ring[(size_t)h * s.ring + at]);
    }
    const int *as = s.act_snd + (size_t)h * s.act_cap, *ar = s.act_rcv + (size_t)h * s.act_cap;
    for (int i = lane; i < hr.n_snd; i += 32)
        prefetch_l1(&s.snd[as[i]].rto_at);
    for (int i = lane; i < hr.n_rcv; i += 32)
        prefetch_l1(&s.rcv[ar[i]].delack_at);
    __syncwarp();
    return staged ? sh.fr : nullptr;
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
#ifdef TB_PROFILE
    unsigned long long sp0 = globaltimer();
#endif
    if (on)
        sw_phase_sizes(x, sh, lane);
    __syncwarp();
    if (lane == 0)
        sw_phase_layout(x, sh);
    __syncwarp();
    sw_phase_copy(x, sh, lane, 32);
    __syncwarp();
    if (on)
        pk = sw_phase_window(x, sh, lane);
    __syncwarp();
    if (x.spray)
    {
        if (sh.staged)
            sw_phase_spray_warp(x, sh, lane, my_ties);
        else if (lane == 0)
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
#ifdef TB_PROFILE
    unsigned long long sp1 = globaltimer();
    if (lane == 0)
        atomicAdd(&s.ctl->prof_phase[6], sp1 - sp0);
#endif
    bool act = false;
    if (on)
        act = sw_phase_egress(x, sh, lane, my_ties, drops, marks, ovf);
    __syncwarp();
#ifdef TB_PROFILE
    if (lane == 0)
        atomicAdd(&s.ctl->prof_phase[7], globaltimer() - sp1);
#endif
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
    extern __shared__ __align__(16) unsigned char dyn_smem[];
    SwShared *sw_sh = reinterpret_cast<SwShared *>(dyn_smem); // one per warp
    __shared__ unsigned blk_act, blk_done;
    __shared__ unsigned long long blk_wake;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int gwarp = blockIdx.x * WARPS_PER_BLOCK + warp, nwarps = gridDim.x * WARPS_PER_BLOCK;
    const int host_units = (s.H + host_lanes - 1) / host_lanes;
    const int units = host_units + s.S;
    SlotCtl *ctl = s.ctl;
    volatile SlotCtl *vc = ctl;
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
        if (vc->finished)
            return;
        const int64_t t = vc->slot;
        unsigned ties = 0;
        for (int u = gwarp; u < units; u += nwarps)
        {
#ifdef TB_PROFILE
            unsigned long long p0 = globaltimer();
#endif
            if (u < host_units)
            {
                int h = u * host_lanes + lane;
                const Frame *stage = nullptr;
                if (host_lanes == 1)
                {
                    h = u;
                    stage = host_prepare(s, h, t, lane, sw_sh[warp]);
                }
                if (lane < host_lanes && h < s.H)
                {
                    int64_t w = INT64_MAX;
                    unsigned done = 0;
                    if (host_step(s, h, t, &w, &ties, &done, stage))
                        atomicOr(&blk_act, 1u);
                    if (done)
                        atomicAdd(&blk_done, done);
                    atomicMin(&blk_wake, (unsigned long long)w);
                }
                __syncwarp(); // (the staging area is reused by the warp's next unit)
            }
            else if (switch_step(s, u - host_units, t, lane, sw_sh[warp], ties) && lane == 0)
                atomicOr(&blk_act, 1u);
#ifdef TB_PROFILE
            if (lane == 0)
                atomicMax(u < host_units ? &ctl->prof_host_max : &ctl->prof_sw_max, globaltimer() - p0);
#endif
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
            unsigned g = ld_gen(&ctl->gen);
            __threadfence();
            unsigned arrived = atomicAdd(&ctl->arrive, 1u) + 1;
            if (arrived == gridDim.x)
            {
                __threadfence();
                vc->arrive = 0;
                unsigned fd = atomicAdd(&ctl->flows_done, 0u);
                if (fd >= (unsigned)s.M || t + 1 >= s.max_slots)
                    vc->finished = 1;
                unsigned cur = atomicAdd(&ctl->act_cur, 0u), prev = vc->act_prev;
                unsigned long long nw = atomicAdd(&ctl->next_wake, 0ull);
                int64_t next = t + 1;
                if (cur == 0 && prev == 0 && nw != ~0ull && (int64_t)nw > next)
                    next = (int64_t)nw < s.max_slots ? (int64_t)nw : s.max_slots;
                vc->act_prev = cur;
                vc->act_cur = 0;
                vc->next_wake = ~0ull;
                vc->slot = next;
                vc->slots_run = vc->slots_run + 1;
#ifdef TB_PROFILE
                unsigned long long now = globaltimer();
                if (vc->prof_release)
                    vc->prof_slot_sum = vc->prof_slot_sum + (now - vc->prof_release);
                vc->prof_release = now;
                vc->prof_host_sum = vc->prof_host_sum + atomicAdd(&ctl->prof_host_max, 0ull);
                vc->prof_sw_sum = vc->prof_sw_sum + atomicAdd(&ctl->prof_sw_max, 0ull);
                vc->prof_host_max = 0;
                vc->prof_sw_max = 0;
#endif
                __threadfence();
                atomicAdd(&ctl->gen, 1u);
            }
            else
            {
                long long spins = 0;
                while (ld_gen(&ctl->gen) == g)
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

// dynamic shared memory of a block: one switch scratch (with its staging area) per warp
constexpr size_t SMEM_BYTES = sizeof(SwShared) * WARPS_PER_BLOCK;

static bool smem_attr()
{
    static bool ok = cudaFuncSetAttribute(slot_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SMEM_BYTES) == cudaSuccess;
    return ok;
}

int slot_kernel_blocks_per_sm()
{
    int n = 0;
    if (!smem_attr() || cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, slot_kernel, WARPS_PER_BLOCK * 32, SMEM_BYTES) != cudaSuccess)
        return 0;
    return n;
}

int launch_slots(const Sim &s, int grid, int max_slots_per_launch, int host_lanes, cudaStream_t stream)
{
    if (!smem_attr())
        return (int)cudaErrorInvalidValue;
    void *args[] = {(void *)&s, (void *)&max_slots_per_launch, (void *)&host_lanes};
    cudaError_t e = cudaLaunchCooperativeKernel((const void *)slot_kernel, dim3(grid), dim3(WARPS_PER_BLOCK * 32), args, SMEM_BYTES, stream);
    return e == cudaSuccess ? 0 : (int)e;
}

} // namespace tb
