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

#include <algorithm>
#include <climits>
#include <cstdint>
#include <cstring>
#include <cuda_runtime.h>

namespace tb
{

constexpr int WARPS_PER_BLOCK = TB_WARPS_PER_BLOCK;
// resident blocks per SM that each instantiation's register budget allows: 4 for several hosts
// per warp (with the smaller staging areas, four blocks fit an SM), 2 for one host per warp (two
// blocks at most fit with its staging areas; more registers spare the host's event loop spills)
constexpr int MIN_BLOCKS_MANY = 4, MIN_BLOCKS_ONE = 2;
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

// the stream's look-ahead rows (tb_common.cuh), in global memory, read through the read-only path
__device__ const RngAhead g_rng_ahead = make_rng_ahead();

// Per-packet spraying's draws with staged frames: the merged arrival order, then the draws. Each
// frame's (time, longer first) is one 32-bit key (its offset in the slot, 21 bits; 2047 - its
// length, 11 bits), so a merge step is one warp-wide minimum of the ports' head keys; frames that tie
// on the key are ordered by lane 0 exactly as the serial merge (sw_phase_spray) orders them, scanning
// the tied ports in port order. The merge only records the order: a prefix over it gives each
// drawing frame its place among the slot's draws, and every draw is then computed at once, from the
// stream's state and the look-ahead rows. Returns false, having written nothing but the warp's
// scratch, when a frame's key does not fit (the argmin merge below then runs). The scratch: the
// windows' flat starts in base (phase 5 writes it afterwards); keys, then places, in the egress
// sources region; the merge order and each frame's draw kind in the egress times region.
__device__ bool sw_spray_keyed(const SwCtx &x, SwShared &sh, int lane, unsigned &ties)
{
    const unsigned FULL = 0xffffffffu;
    const int k = x.sr->k;
    const WorldDesc &wd = *x.wd;
    const int64_t S0 = x.t * SLOT_PS;
    const Input in = input_of(x, sh, lane < k ? lane : 0);
    const int c = lane < k ? in.count() : 0;
    int incl = c;
    for (int o = 1; o < 32; o <<= 1)
    {
        const int v = __shfl_up_sync(FULL, incl, o);
        if (lane >= o)
            incl += v;
    }
    const int total = __shfl_sync(FULL, incl, 31), base = incl - c;
    if (total == 0)
        return true;
    if (total > RNG_AHEAD)
        return false;
    uint32_t *key = sh.eref();                            // [total]: keys, then places
    int *ord = reinterpret_cast<int *>(sh.ets());         // [total]: flat frames in merge order
    int *kind = reinterpret_cast<int *>(sh.ets()) + sh.cap; // [total]: 0 port down, 1 no routes (0 written), nr + 1
    if (lane < k)
        sh.base[lane] = base;
    bool bad = false;
    for (int j = 0; j < c; j++)
    {
        const Frame &f = *in.at(j);
        const int64_t off = f.ts - S0;
        bad |= off < 0 || off >= (1 << 21) || f.len > 2047;
        key[base + j] = (uint32_t)off << 11 | (uint32_t)(2047 - f.len);
        const int ep = wd.n_fail ? epoch_of(wd, f.ts) : 0;
        kind[base + j] = port_down(wd, x.sr->local, lane, ep) ? 0 : 1 + routes_to(wd, x.sr->local, f.dst, ep);
    }
    if (__any_sync(FULL, bad))
        return false;
    __syncwarp();
    int pos = 0;
    uint32_t head = c ? key[base] : 0xFFFFFFFFu;
    for (int r = 0; r < total; r++)
    {
        const uint32_t m = __reduce_min_sync(FULL, head);
        const unsigned cand = __ballot_sync(FULL, head == m);
        int best = __ffs(cand) - 1;
        if (cand & (cand - 1))
        {
            // equal times and lengths: the upstream chains, then the connection id
            const Frame *bf = nullptr;
            for (unsigned cc = cand; cc; cc &= cc - 1)
            {
                const int q = __ffs(cc) - 1;
                const int pq = __shfl_sync(FULL, pos, q);
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
        if (lane == best)
        {
            ord[r] = base + pos;
            pos++;
            head = pos < c ? key[base + pos] : 0xFFFFFFFFu;
        }
    }
    __syncwarp();
    // places among the draws: an exclusive prefix of the drawing frames in merge order
    int run = 0;
    for (int r0 = 0; r0 < total; r0 += 32)
    {
        const int r = r0 + lane, i = r < total ? ord[r] : 0, v = r < total && kind[i] >= 2;
        int sc = v;
        for (int o = 1; o < 32; o <<= 1)
        {
            const int u = __shfl_up_sync(FULL, sc, o);
            if (lane >= o)
                sc += u;
        }
        if (r < total)
            key[i] = run + sc - v;
        run += __shfl_sync(FULL, sc, 31);
    }
    __syncwarp();
    const Rng st = x.s->sw_rng[x.sw];
    for (int i = lane; i < total; i += 32)
    {
        const int v = kind[i];
        if (v == 0)
            continue;
        int q = 0;
        while (q + 1 < k && sh.base[q + 1] <= i)
            q++;
        uint8_t u = 0;
        if (v >= 2)
        {
            const uint32_t *row = g_rng_ahead.r[key[i] + 1];
            u = (uint8_t)int_of_u01(u01_of(rng_ahead_value<RNG_M1>(row, st.s), rng_ahead_value<RNG_M2>(row + 3, st.s + 3)), (uint32_t)(v - 1));
        }
        x.s->sw_up[x.scratch + (size_t)q * 2 * MAX_TX + (i - sh.base[q])] = u;
    }
    // the stream after the slot's draws: each component's last three values
    __syncwarp(); // (every lane has read the stream)
    if (lane < 6)
    {
        const int cmp = lane / 3, m = run - 2 + lane % 3;
        const uint32_t *row = g_rng_ahead.r[m > 0 ? m : 1] + 3 * cmp;
        x.s->sw_rng[x.sw].s[lane] = m <= 0 ? st.s[3 * cmp + m + 2]
                                           : (cmp ? rng_ahead_value<RNG_M2>(row, st.s + 3) : rng_ahead_value<RNG_M1>(row, st.s));
    }
    return true;
}

// Per-packet spraying's draws with staged frames whose keys do not fit (sw_spray_keyed): the merged
// arrival order by a warp-wide argmin of (time, length), one draw after another.
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

// The world's rule for this slot (reference src/kernel.cuh:79-112, per world): the next launch
// slot its entities run, and its time origin; both read through L2 (the controller of another SM
// writes them)
__device__ __forceinline__ int64_t world_next(const Sim &s, int w) { return __ldcg(&s.wctl[w].next); }
__device__ __forceinline__ int64_t world_t0(const Sim &s, int w) { return __ldcg(&s.wctl[w].t0); }

// a host's slot results into its world's record (wake: a world-local slot)
__device__ __forceinline__ void host_report(const Sim &s, int w, int64_t t0, bool act, int64_t wake, unsigned done)
{
    WorldCtl *wc = &s.wctl[w];
    if (act)
        atomicOr(&wc->act, 1u);
    if (wake != INT64_MAX)
        atomicMin(&wc->wake, (unsigned long long)(wake + t0));
    if (done)
        atomicAdd(&wc->fdone, done);
}

// host_step's timer scan on the whole warp: the timers of the host's active connections due before
// E0, in host_step's order (senders' retransmission then SYN timers, then receivers' delayed-ACK,
// SYN, last-ACK and FIN timers, each list in its order), the first DUE_CAP of them into `due`; the
// count kept is returned (every lane), the count left out goes to *ovf.
__device__ int collect_due_warp(const Sim &s, const HostRec &hr, int h, int64_t E0, int lane, Due *due, int *ovf)
{
    const unsigned FULL = 0xffffffffu;
    const int *as = s.act_snd + (size_t)h * s.act_cap, *ar = s.act_rcv + (size_t)h * s.act_cap;
    const int ns = hr.n_snd, nr = hr.n_rcv;
    int n = 0;
    auto place = [&](int cnt) {
        int incl = cnt;
        for (int o = 1; o < 32; o <<= 1)
        {
            const int v = __shfl_up_sync(FULL, incl, o);
            if (lane >= o)
                incl += v;
        }
        const int at = n + incl - cnt;
        n += __shfl_sync(FULL, incl, 31);
        return at;
    };
    for (int i0 = 0; i0 < ns; i0 += 32)
    {
        const int i = i0 + lane;
        int f = 0;
        int64_t v[2] = {-1, -1};
        if (i < ns)
        {
            f = as[i];
            v[0] = s.snd[f].rto_at;
            v[1] = s.snd[f].syn_at;
        }
        const int kinds[2] = {0, 2};
        int at = place((v[0] >= 0 && v[0] < E0) + (v[1] >= 0 && v[1] < E0));
        for (int j = 0; j < 2; j++)
            if (v[j] >= 0 && v[j] < E0)
            {
                if (at < DUE_CAP)
                    due[at] = {v[j], f, kinds[j]};
                at++;
            }
    }
    for (int i0 = 0; i0 < nr; i0 += 32)
    {
        const int i = i0 + lane;
        int f = 0;
        int64_t v[4] = {-1, -1, -1, -1};
        if (i < nr)
        {
            f = ar[i];
            const RcvRec &R = s.rcv[f];
            v[0] = R.delack_at;
            v[1] = R.syn_at;
            v[2] = R.last_at;
            v[3] = R.frx_at;
        }
        const int kinds[4] = {1, 3, 4, 5};
        int cnt = 0;
        for (int j = 0; j < 4; j++)
            cnt += v[j] >= 0 && v[j] < E0;
        int at = place(cnt);
        for (int j = 0; j < 4; j++)
            if (v[j] >= 0 && v[j] < E0)
            {
                if (at < DUE_CAP)
                    due[at] = {v[j], f, kinds[j]};
                at++;
            }
    }
    *ovf = n > DUE_CAP ? n - DUE_CAP : 0;
    return n < DUE_CAP ? n : DUE_CAP;
}

// host_step's last phase on the whole warp: the host's finished connections leave its active
// lists (the others keep their order; lanes read a chunk of 32 entries, then write the kept ones
// back at or below it) and the earliest timer of the connections that stay is returned (every
// lane). The host's lists and counts are those its lane 0 has just written.
__device__ int64_t prune_lists_warp(const Sim &s, int h, int lane)
{
    const unsigned FULL = 0xffffffffu, below = (1u << lane) - 1;
    HostRec &hr = s.hosts[h];
    int *as = s.act_snd + (size_t)h * s.act_cap, *ar = s.act_rcv + (size_t)h * s.act_cap;
    int64_t next = INT64_MAX;
    const int ns = hr.n_snd, nr = hr.n_rcv;
    int k = 0;
    for (int i0 = 0; i0 < ns; i0 += 32)
    {
        const int i = i0 + lane;
        int f = 0;
        bool keep = false;
        if (i < ns)
        {
            f = as[i];
            const SndRec &S = s.snd[f];
            keep = S.st != S_DONE;
            if (keep && S.rto_at >= 0 && S.rto_at < next)
                next = S.rto_at;
            if (keep && S.syn_at >= 0 && S.syn_at < next)
                next = S.syn_at;
        }
        const unsigned m = __ballot_sync(FULL, keep);
        __syncwarp(); // (every lane has read its entry)
        if (keep)
            as[k + __popc(m & below)] = f;
        k += __popc(m);
    }
    const int ks = k;
    k = 0;
    for (int i0 = 0; i0 < nr; i0 += 32)
    {
        const int i = i0 + lane;
        int f = 0;
        bool keep = false;
        if (i < nr)
        {
            f = ar[i];
            const RcvRec &R = s.rcv[f];
            keep = !rcv_idle_for_good(R);
            if (keep)
            {
                const int64_t v[4] = {R.delack_at, R.syn_at, R.last_at, R.frx_at};
                for (int j = 0; j < 4; j++)
                    if (v[j] >= 0 && v[j] < next)
                        next = v[j];
            }
        }
        const unsigned m = __ballot_sync(FULL, keep);
        __syncwarp();
        if (keep)
            ar[k + __popc(m & below)] = f;
        k += __popc(m);
    }
    for (int o = 16; o > 0; o >>= 1)
    {
        const int64_t v = __shfl_xor_sync(FULL, next, o);
        next = v < next ? v : next;
    }
    __syncwarp(); // (every lane has read the counts)
    if (lane == 0)
    {
        hr.n_snd = ks;
        hr.n_rcv = k;
    }
    return next;
}

// A host unit at launch slot t: one host per warp (host_lanes 1) or one per lane. With one host
// per warp, the warp reads the host's link-message tags (by launch slot) together with its world's
// rule; a host whose world does not run this slot, or that has no frame arriving, no timer due and
// an empty queue, only reports its wake-up. Otherwise the warp copies the host's incoming link
// messages to shared memory (one cooperative pass) and prefetches into L1 what the host's events
// will read: the records of the frames' connections with the heads of their sent lists and RTT
// histories, the head frames of the host's egress queue, and the timers of its active
// connections; then lane 0 runs the host's slot (host_step) on the staged frames, or in place
// when they do not fit. With several hosts per warp each lane runs its own host in place: the
// unit's hosts are h0 .. h0 + nh - 1. Flows completed are added to *done_sink.
template <bool MANY>
__device__ __forceinline__ void host_unit(const Sim &s, int h0, int nh, int64_t t, int lane, SwShared &sh, unsigned &ties,
                                          unsigned *done_sink)
{
    int h, w = 0, n2 = -1, n1 = -1, due_n = 0, due_ovf = 0;
    int64_t t0 = 0;
    bool run = false;
    const Frame *stage = nullptr;
    Due *due = nullptr;
    if constexpr (!MANY)
    {
        h = h0;
        const HostRec &hr = s.hosts[h];
        w = hr.world;
        const int link = hr.in_link;
        n2 = t >= 2 ? msg_count(s, t - 2, link) : 0;
        n1 = t >= 1 ? msg_count(s, t - 1, link) : 0;
        const int n = n2 + n1;
        const int64_t next = world_next(s, w);
        t0 = world_t0(s, w);
        if (t < next)
            return;
        if (n == 0 && t - t0 < hr.wake && hr.q_size == 0)
        {
            if (lane == 0 && hr.wake != INT64_MAX)
                atomicMin(&s.wctl[w].wake, (unsigned long long)(hr.wake + t0));
            return;
        }
        const bool staged = n <= sh.cap;
        if (staged)
            for (int i = lane; i < n; i += 32)
                frame_load_link(sh.fr()[i], i < n2 ? msg_frames(s, t - 2, link) + i : msg_frames(s, t - 1, link) + (i - n2));
        __syncwarp();
        if (staged)
            for (int i = lane; i < n; i += 32)
            {
                const Frame &f = sh.fr()[i];
                if (f.to_sender)
                {
                    const SndRec *S = &s.snd[f.flow];
                    for (int b = 0; b < (int)sizeof(SndRec); b += 128)
                        prefetch_l1((const char *)S + b);
                    const uint64_t off = S->it_off;
                    prefetch_l1(&s.it_start[off + S->it_head]);
                    prefetch_l1(&s.it_fl[off + 4 * (S->it_head >> 3)]); // (the flag word of the head's eight)
                    const uint32_t hh = S->h_head;
                    prefetch_l1(&s.h_seq[off + hh]);
                    prefetch_l1(&s.h_end[off + hh]);
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
        if (sh.cap * (int)(sizeof(int64_t) + sizeof(uint32_t)) >= DUE_CAP * (int)sizeof(Due))
        {
            due = reinterpret_cast<Due *>(sh.ets()); // (the egress regions, unused by a host)
            due_n = collect_due_warp(s, hr, h, (t - t0 + 1) * SLOT_PS, lane, due, &due_ovf);
        }
        else
        {
            const int *as = s.act_snd + (size_t)h * s.act_cap, *ar = s.act_rcv + (size_t)h * s.act_cap;
            for (int i = lane; i < hr.n_snd; i += 32)
                prefetch_l1(&s.snd[as[i]].rto_at);
            for (int i = lane; i < hr.n_rcv; i += 32)
                prefetch_l1(&s.rcv[ar[i]].delack_at);
        }
        __syncwarp();
        stage = staged ? sh.fr() : nullptr;
        run = lane == 0;
    }
    else
    {
        h = h0 + lane;
        if (lane < nh)
        {
            const HostRec &hr = s.hosts[h];
            w = hr.world;
            t0 = world_t0(s, w);
            run = t >= world_next(s, w);
            if (run)
            {
                // all lanes at once: the tags of the host's link messages, then the records of
                // the connections of its first arrivals into L1 (the lanes' event loops diverge
                // next, and would each wait for these one after the other)
                const int link = hr.in_link;
                n2 = t >= 2 ? msg_count(s, t - 2, link) : 0;
                n1 = t >= 1 ? msg_count(s, t - 1, link) : 0;
                const Frame *m2 = msg_frames(s, t - 2, link), *m1 = msg_frames(s, t - 1, link);
                for (int j = 0; j < 4 && j < n2 + n1; j++)
                {
                    const Frame *f = j < n2 ? &m2[j] : &m1[j - n2];
                    const uint32_t flow = __ldcg(&f->flow);
                    const uint8_t to_snd = __ldcg(&f->to_sender);
                    prefetch_l1(to_snd ? (const void *)&s.snd[flow] : (const void *)&s.rcv[flow]);
                }
                if (hr.q_size > 0)
                    prefetch_l1(&s.host_ring[(size_t)h * s.ring + hr.q_head]);
            }
        }
    }
    int64_t wake = INT64_MAX;
    unsigned done = 0;
    bool act = false;
    if (run)
    {
        act = host_step(s, h, t - t0, t, &wake, &ties, &done, stage, n2, n1, !MANY, due, due_n, due_ovf);
        if constexpr (MANY)
            host_report(s, w, t0, act, wake, done);
    }
    if constexpr (!MANY)
    {
        // the whole warp prunes the host's active lists; the earliest timer left bounds the wake-up
        __syncwarp();
        const int64_t nt = prune_lists_warp(s, h, lane);
        if (lane == 0)
        {
            HostRec &hr = s.hosts[h];
            if (hr.q_size == 0 && nt != INT64_MAX && nt / SLOT_PS < hr.wake)
                hr.wake = nt / SLOT_PS;
            host_report(s, w, t0, act, hr.wake, done);
        }
    }
    if (run && done)
        atomicAdd(done_sink, done);
    __syncwarp(); // (the staging area is reused by the warp's next unit)
}

// one switch, one slot (launch slot gt), by its warp (lanes >= k idle but take part in the warp
// barriers); nothing when its world does not run this slot
template <bool PORT_LOCAL>
__device__ bool switch_step(const Sim &s, int sw, int64_t gt, int lane, SwShared &sh, unsigned &ties)
{
    const SwRec &sr = s.sws[sw];
    const int64_t next = world_next(s, sr.world), t0 = world_t0(s, sr.world);
    const int64_t t = gt - t0;
    SwCtx x;
    x.s = &s;
    x.wd = &s.worlds[sr.world];
    x.sr = &sr;
    x.sw = sw;
    x.ports = s.ports + sr.port0;
    x.scratch = (size_t)sw * s.kmax * 2 * MAX_TX;
    x.t = t;
    x.gt = gt;
    x.spray = x.wd->spray != 0;
    const int k = sr.k;
    const bool on = lane < k;
    unsigned pk = 0, drops = 0, marks = 0, ovf = 0, my_ties = 0;
#ifdef TB_PROFILE
    unsigned long long sp0 = globaltimer();
#endif
    if (on)
        sw_phase_sizes(x, sh, lane);
    // its world does not run this slot; or no frame arriving and every queue empty: nothing to do
    // (its link messages of this slot stay unwritten, and a stale tag reads as an empty message)
    if (gt < next || !__any_sync(0xffffffffu, on && (sh.raw2[lane] | sh.raw1[lane] | x.ports[lane].q_size) != 0))
        return false;
    __syncwarp();
    if (lane == 0)
        sw_phase_layout(x, sh);
    __syncwarp();
    sw_phase_copy(x, sh, lane, 32);
    __syncwarp();
    if (on)
        pk = sw_phase_window(x, sh, lane);
    __syncwarp();
#ifdef TB_PROFILE
    unsigned long long sp2 = globaltimer();
    if (lane == 0)
        atomicAdd(&s.ctl->prof_phase[11], sp2 - sp0);
#endif
    if (x.spray)
    {
        if (sh.staged)
        {
            const bool keyed = sw_spray_keyed(x, sh, lane, my_ties);
#ifdef TB_PROFILE
            if (lane == 0)
                atomicAdd(&s.ctl->prof_phase[keyed ? 13 : 14], 1000ull);
#endif
            if (!keyed)
                sw_phase_spray_warp(x, sh, lane, my_ties);
        }
        else if (lane == 0)
            sw_phase_spray(x, sh, my_ties);
        __syncwarp();
    }
#ifdef TB_PROFILE
    unsigned long long sp3 = globaltimer();
    if (lane == 0)
        atomicAdd(&s.ctl->prof_phase[12], sp3 - sp2);
#endif
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
        act = sw_phase_egress<PORT_LOCAL>(x, sh, lane, my_ties, drops, marks, ovf);
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

// PORT_LOCAL: switch ports keep the slot's transmission chain and last enqueued frame in shared
// memory (PortEgress); MIN_BLOCKS: the register budget. Separate instantiations, chosen per launch.
template <bool PORT_LOCAL, int MIN_BLOCKS>
__global__ void __launch_bounds__(WARPS_PER_BLOCK * 32, MIN_BLOCKS) slot_kernel(Sim s, int max_slots_per_launch, int host_lanes, int stage_cap)
{
    extern __shared__ __align__(16) unsigned char dyn_smem[];
    __shared__ unsigned blk_done;
    __shared__ int blk_last;
    __shared__ unsigned long long blk_next;
    __shared__ unsigned blk_alive;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int gwarp = blockIdx.x * WARPS_PER_BLOCK + warp, nwarps = gridDim.x * WARPS_PER_BLOCK;
    const int host_units = (s.H + host_lanes - 1) / host_lanes;
    const int units = host_units + s.S;
    SwShared &sh = *sw_shared_at(dyn_smem + (size_t)warp * sw_shared_bytes(stage_cap, PORT_LOCAL), stage_cap); // the warp's scratch
    __syncwarp();
    SlotCtl *ctl = s.ctl;
    volatile SlotCtl *vc = ctl;
    for (int it = 0; it < max_slots_per_launch; it++)
    {
        if (threadIdx.x == 0)
            blk_done = 0;
        __syncthreads();
        // (written by the last block of the previous barrier, before it released the others)
        if (vc->finished)
            return;
        const int64_t t = vc->slot;
        unsigned ties = 0;
        const int n_iter = s.unit_list ? s.n_list : units;
        for (int i = gwarp; i < n_iter; i += nwarps)
        {
            const int u = s.unit_list ? __ldg(&s.unit_list[i]) : i;
#ifdef TB_PROFILE
            unsigned long long p0 = globaltimer();
#endif
            if (u < host_units)
            {
                const int h0 = u * host_lanes;
                host_unit<MIN_BLOCKS == MIN_BLOCKS_MANY>(s, h0, min(host_lanes, s.H - h0), t, lane, sh, ties, &blk_done);
            }
            else
            {
                const int sw = u - host_units;
                if (switch_step<PORT_LOCAL>(s, sw, t, lane, sh, ties) && lane == 0)
                    atomicOr(&s.wctl[s.sws[sw].world].act, 1u);
            }
#ifdef TB_PROFILE
            if (lane == 0)
                atomicMax(u < host_units ? &ctl->prof_host_max : &ctl->prof_sw_max, globaltimer() - p0);
#endif
        }
        __syncthreads();
        unsigned g = 0; // (thread 0: the barrier generation before it arrives)
        if (threadIdx.x == 0)
        {
            if (blk_done)
                atomicAdd(&ctl->flows_done, blk_done);
            blk_next = ~0ull;
            blk_alive = 0;
            // grid barrier: the last block to arrive ends the slot and releases the others
            g = ld_gen(&ctl->gen);
            __threadfence();
            unsigned arrived = atomicAdd(&ctl->arrive, 1u) + 1;
            blk_last = arrived == gridDim.x;
        }
        __syncthreads();
        if (blk_last)
        {
            __threadfence();
            // every world's next slot: finished worlds stop; a world where nothing was sent in
            // this or the previous slot skips to its earliest wake-up
            for (int w = threadIdx.x; w < s.W; w += blockDim.x)
            {
                WorldCtl *wc = &s.wctl[w];
                volatile WorldCtl *vw = wc;
                int64_t nx = vw->next;
                if (nx == INT64_MAX)
                    continue;
                const unsigned cur = atomicExch(&wc->act, 0u), prev = vw->prev;
                const unsigned long long wake = atomicExch(&wc->wake, (unsigned long long)INT64_MAX);
                vw->prev = cur;
                if (t >= nx)
                {
                    if (atomicAdd(&wc->fdone, 0u) >= (unsigned)s.worlds[w].n_msgs)
                    {
                        vw->next = INT64_MAX;
                        continue;
                    }
                    nx = (cur == 0 && prev == 0 && (int64_t)wake > t + 1) ? (int64_t)wake : t + 1;
                    vw->next = nx;
                }
                atomicMin(&blk_next, (unsigned long long)nx);
                atomicAdd(&blk_alive, 1u);
            }
            __syncthreads();
            if (threadIdx.x == 0)
            {
                vc->arrive = 0;
                int64_t next = (int64_t)blk_next;
                if (next > s.max_slots)
                    next = s.max_slots;
                if (blk_alive == 0)
                    next = t + 1; // (finished: nothing left to skip to)
                if (blk_alive == 0 || t + 1 >= s.max_slots)
                    vc->finished = 1;
                vc->slot = next > t + 1 ? next : t + 1;
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
        }
        else if (threadIdx.x == 0)
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
        if (threadIdx.x == 0)
            __threadfence();
        __syncthreads();
    }
}


// ------------------------------------------------------------------ batches without a grid barrier
// A batch's worlds are independent: each runs its own slots on a barrier of its own, so that a
// slot of one world waits only for that world's units, not for the slowest unit of the batch.
// The launch's unit list holds host units (first host h < H; up to host_lanes hosts of one world)
// and switches (H + switch). A warp cycles over its units and runs every one whose world runs a
// slot the unit has not done; the unit's lane 0, after the warp, counts it in its world's
// `arrive`, and the world's last unit closes the slot: the world's slot rule (finish, the exact
// idle skip), then the next slot is published (or the world parks: its slot budget for this
// launch is spent, or it is done). A warp whose units are all parked leaves; one that finds
// nothing to run waits (bounded) for its worlds to move.

// the world's slot t is done by all its units: its next slot, or parked (by the unit's lane 0)
__device__ void world_close(const Sim &s, int w, int64_t t)
{
    WorldCtl *wc = &s.wctl[w];
    volatile WorldCtl *vw = wc;
    __threadfence();
    const unsigned cur = atomicExch(&wc->act, 0u), prev = vw->prev;
    const unsigned long long wake = atomicExch(&wc->wake, (unsigned long long)INT64_MAX);
    vw->prev = cur;
    vw->last = t;
    int64_t nx;
    if (atomicAdd(&wc->fdone, 0u) >= (unsigned)s.worlds[w].n_msgs)
        nx = INT64_MAX;
    else
    {
        nx = (cur == 0 && prev == 0 && (int64_t)wake > t + 1) ? (int64_t)wake : t + 1;
        if (nx >= s.max_slots)
        {
            nx = INT64_MAX; // (the run ends at max_slots with flows unfinished, as the batch's does)
            vw->last = s.max_slots - 1;
        }
    }
    atomicAdd((unsigned long long *)&s.ctl->slots_run, 1ull);
    const unsigned budget = vw->budget - 1;
    vw->budget = budget;
    vw->next = nx;
    vw->arrive = 0;
    __threadfence();
    vw->run = (nx == INT64_MAX || budget == 0) ? RUN_PARKED : nx;
}

// before a launch: every world runs from its next slot with a budget; every unit has done nothing
__global__ void free_open(Sim s, unsigned budget)
{
    const int stride = gridDim.x * blockDim.x;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < s.n_list; i += stride)
        s.unit_done[i] = RUN_PARKED;
    for (int w = blockIdx.x * blockDim.x + threadIdx.x; w < s.W; w += stride)
    {
        WorldCtl &c = s.wctl[w];
        c.arrive = 0;
        c.units = s.w_units[w];
        c.budget = budget;
        c.run = c.next == INT64_MAX || c.units == 0 ? RUN_PARKED : c.next;
    }
}

template <bool PORT_LOCAL, int MIN_BLOCKS>
__global__ void __launch_bounds__(WARPS_PER_BLOCK * 32, MIN_BLOCKS) free_kernel(Sim s, int host_lanes, int stage_cap)
{
    extern __shared__ __align__(16) unsigned char dyn_smem[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int gwarp = blockIdx.x * WARPS_PER_BLOCK + warp, nwarps = gridDim.x * WARPS_PER_BLOCK;
    SwShared &sh = *sw_shared_at(dyn_smem + (size_t)warp * sw_shared_bytes(stage_cap, PORT_LOCAL), stage_cap); // the warp's scratch
    __syncwarp();
    const unsigned FULL = 0xffffffffu;
    long long idle = 0;
    for (;;)
    {
        bool live = false, ran = false;
        for (int i = gwarp; i < s.n_list; i += nwarps)
        {
            const int v = __ldg(&s.unit_list[i]);
            const bool host = v < s.H;
            const int w = host ? s.hosts[v].world : s.sws[v - s.H].world;
            int64_t t = 0, done = 0;
            if (lane == 0)
            {
                t = __ldcg(&s.wctl[w].run);
                done = s.unit_done[i];
            }
            t = __shfl_sync(FULL, t, 0);
            done = __shfl_sync(FULL, done, 0);
            if (t == RUN_PARKED)
                continue;
            live = true;
            if (done == t)
                continue; // (done; its world's other units are not)
            ran = true;
            __threadfence(); // (what the world's units wrote in its last slot, before `run` moved)
            unsigned ties = 0;
            if (host)
            {
                const WorldDesc &wd = s.worlds[w];
                host_unit<MIN_BLOCKS == MIN_BLOCKS_MANY>(s, v, min(host_lanes, wd.host0 + wd.H1 - v), t, lane, sh, ties,
                                                         &s.ctl->flows_done);
            }
            else if (switch_step<PORT_LOCAL>(s, v - s.H, t, lane, sh, ties) && lane == 0)
                atomicOr(&s.wctl[w].act, 1u);
            __syncwarp();
            if (lane == 0)
            {
                s.unit_done[i] = t;
                __threadfence();
                if (atomicAdd(&s.wctl[w].arrive, 1u) + 1 == __ldcg(&s.wctl[w].units))
                    world_close(s, w, t);
            }
            __syncwarp();
        }
        if (!live)
            return;
        if (ran)
        {
            idle = 0;
            continue;
        }
        if (++idle > BARRIER_SPIN_LIMIT || __ldcg(&s.ctl->error))
        {
            if (lane == 0 && idle > BARRIER_SPIN_LIMIT)
            {
                atomicExch(&s.ctl->error, 1);
                atomicAdd(&s.ev[EV_BARRIER_TIMEOUT], 1ull);
            }
            return;
        }
        __nanosleep(64);
    }
}

// dynamic shared memory of a block: one switch scratch (with its staging area) per warp
static size_t smem_bytes(int stage_cap, bool port_local) { return sw_shared_bytes(stage_cap, port_local) * WARPS_PER_BLOCK; }

// the instantiation of a launch shape: several hosts per warp, one host per warp, one host per
// warp with port-local switch egress; each with the grid barrier or without (F_*: batches)
enum
{
    K_MANY,
    K_ONE,
    K_ONE_PL,
    F_MANY,
    F_ONE,
    F_ONE_PL,
    K_N
};
static int kind_of(int host_lanes, bool port_local, bool free = false)
{
    return (host_lanes > 1 ? K_MANY : port_local ? K_ONE_PL : K_ONE) + (free ? F_MANY : 0);
}
static const void *kernel_of(int k)
{
    switch (k)
    {
    case K_MANY:
        return (const void *)slot_kernel<false, MIN_BLOCKS_MANY>;
    case K_ONE:
        return (const void *)slot_kernel<false, MIN_BLOCKS_ONE>;
    case K_ONE_PL:
        return (const void *)slot_kernel<true, MIN_BLOCKS_ONE>;
    case F_MANY:
        return (const void *)free_kernel<false, MIN_BLOCKS_MANY>;
    case F_ONE:
        return (const void *)free_kernel<false, MIN_BLOCKS_ONE>;
    default:
        return (const void *)free_kernel<true, MIN_BLOCKS_ONE>;
    }
}

static bool smem_attr(int k)
{
    static bool ok[K_N], tried[K_N];
    if (!tried[k])
    {
        tried[k] = true;
        const bool pl = k == K_ONE_PL || k == F_ONE_PL;
        ok[k] = cudaFuncSetAttribute(kernel_of(k), cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_bytes(SW_STAGE_MAX, pl)) == cudaSuccess;
    }
    return ok[k];
}

// The preferred shared-memory carveout, in percent of the SM's maximum: the shared memory of the
// blocks a launch puts on one SM and no more, so that the rest of the SM's unified L1 / shared
// memory is L1, where the units' records, ring heads and prefetched lines stay between slots.
static int carveout[K_N] = {-1, -1, -1, -1, -1, -1}; // the last ones set (-1: none)
static void set_carveout(int k, int pct)
{
    if (pct != carveout[k] && cudaFuncSetAttribute(kernel_of(k), cudaFuncAttributePreferredSharedMemoryCarveout, pct) == cudaSuccess)
        carveout[k] = pct;
}

int slot_kernel_blocks_per_sm(int stage_cap, bool port_local, int host_lanes, bool free)
{
    int n = 0;
    port_local = port_local && host_lanes == 1;
    const int k = kind_of(host_lanes, port_local, free);
    if (stage_cap < 1 || stage_cap > SW_STAGE_MAX || !smem_attr(k))
        return 0;
    set_carveout(k, 100); // (occupancy with all of the shared memory)
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kernel_of(k), WARPS_PER_BLOCK * 32, smem_bytes(stage_cap, port_local)) != cudaSuccess)
        return 0;
    return n;
}

// a cooperative launch of kernel kind k (all its blocks resident: the waits need it)
static int launch_kind(int k, void **args, int grid, int stage_cap, bool port_local, cudaStream_t stream)
{
    int dev = 0, sms = 1, max_smem = 1;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaDeviceGetAttribute(&max_smem, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev);
    const long long per_sm = (grid + sms - 1) / sms;
    const size_t bytes = smem_bytes(stage_cap, port_local);
    const long long need = per_sm * (long long)(bytes + 2048); // (+ the block's reserved and static shared memory)
    set_carveout(k, (int)std::min<long long>(100, (need * 100 + max_smem - 1) / max_smem));
    cudaError_t e = cudaLaunchCooperativeKernel(kernel_of(k), dim3(grid), dim3(WARPS_PER_BLOCK * 32), args, bytes, stream);
    if (e == cudaErrorCooperativeLaunchTooLarge)
    {
        // (the carveout left too little shared memory for the blocks to be resident at once)
        cudaGetLastError();
        set_carveout(k, 100);
        e = cudaLaunchCooperativeKernel(kernel_of(k), dim3(grid), dim3(WARPS_PER_BLOCK * 32), args, bytes, stream);
    }
    return e == cudaSuccess ? 0 : (int)e;
}

int launch_slots(const Sim &s, int grid, int max_slots_per_launch, int host_lanes, int stage_cap, bool port_local, cudaStream_t stream)
{
    port_local = port_local && host_lanes == 1; // (several hosts per warp: the plain egress)
    const int k = kind_of(host_lanes, port_local);
    if (!smem_attr(k) || stage_cap < 1 || stage_cap > SW_STAGE_MAX)
        return (int)cudaErrorInvalidValue;
    void *args[] = {(void *)&s, (void *)&max_slots_per_launch, (void *)&host_lanes, (void *)&stage_cap};
    return launch_kind(k, args, grid, stage_cap, port_local, stream);
}

int launch_free(const Sim &s, int grid, int slots_per_world, int host_lanes, int stage_cap, bool port_local, cudaStream_t stream)
{
    port_local = port_local && host_lanes == 1;
    const int k = kind_of(host_lanes, port_local, true);
    if (!smem_attr(k) || stage_cap < 1 || stage_cap > SW_STAGE_MAX || !s.unit_list || !s.unit_done || !s.w_units || slots_per_world < 1)
        return (int)cudaErrorInvalidValue;
    const int n = std::max(s.n_list, s.W);
    free_open<<<(n + 255) / 256, 256, 0, stream>>>(s, (unsigned)slots_per_world);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess)
        return (int)e;
    void *args[] = {(void *)&s, (void *)&host_lanes, (void *)&stage_cap};
    return launch_kind(k, args, grid, stage_cap, port_local, stream);
}

// A launch as a CUDA graph: the launch is captured once per shape, slot count and unit list and
// replayed as a graph; where capturing or instantiating fails, plain launches follow for good.
// free: the batch kernel without a grid barrier (launch_free), with its opening kernel.
int launch_slots_graph(SlotGraph &g, const Sim &s, int grid, int max_slots_per_launch, int host_lanes, int stage_cap, bool port_local,
                       cudaStream_t stream, bool free)
{
    const unsigned long long key[9] = {(unsigned long long)grid, (unsigned long long)max_slots_per_launch, (unsigned long long)host_lanes,
                                       (unsigned long long)stage_cap, (unsigned long long)port_local, (unsigned long long)(uintptr_t)s.unit_list,
                                       (unsigned long long)s.n_list, (unsigned long long)s.max_slots, (unsigned long long)free};
    auto go = [&]() {
        return free ? launch_free(s, grid, max_slots_per_launch, host_lanes, stage_cap, port_local, stream)
                    : launch_slots(s, grid, max_slots_per_launch, host_lanes, stage_cap, port_local, stream);
    };
    if (g.broken)
        return go();
    if (!g.exec || memcmp(key, g.key, sizeof key) != 0)
    {
        if (g.exec)
            cudaGraphExecDestroy((cudaGraphExec_t)g.exec);
        g.exec = nullptr;
        cudaGraph_t graph = nullptr;
        cudaGraphExec_t exec = nullptr;
        int e = 1;
        if (cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal) == cudaSuccess)
        {
            e = go();
            if (cudaStreamEndCapture(stream, &graph) != cudaSuccess)
                e = 1;
        }
        if (e == 0 && graph && cudaGraphInstantiate(&exec, graph, 0) == cudaSuccess)
        {
            g.exec = exec;
            memcpy(g.key, key, sizeof key);
        }
        if (graph)
            cudaGraphDestroy(graph);
        if (!g.exec)
        {
            cudaGetLastError(); // (the failed capture's error)
            g.broken = true;
            return go();
        }
    }
    g.replays++;
    return cudaGraphLaunch((cudaGraphExec_t)g.exec, stream) == cudaSuccess ? 0 : (int)cudaGetLastError();
}

void release_graph(SlotGraph &g)
{
    if (g.exec)
        cudaGraphExecDestroy((cudaGraphExec_t)g.exec);
    g.exec = nullptr;
}

} // namespace tb
