// twins-b200: frame moves and the egress port (a point-to-point device: one-packet device queue
// under a RED queue disc), used by hosts and switch ports.
#pragma once
#include "tb_state.cuh"

namespace tb
{

// Frames that cross entities (link messages) move through L2 only: readers in later slots run
// on other SMs, whose L1 would otherwise hold stale lines (the persistent kernel is never
// relaunched between slots).
TB_D void frame_copy(Frame *d, const Frame *s)
{
    const uint4 *a = reinterpret_cast<const uint4 *>(s);
    uint4 *b = reinterpret_cast<uint4 *>(d);
    uint4 v[FRAME_WORDS];
#pragma unroll
    for (int i = 0; i < FRAME_WORDS; i++)
        v[i] = a[i];
#pragma unroll
    for (int i = 0; i < FRAME_WORDS; i++)
        b[i] = v[i];
}
TB_D void frame_load_link(Frame &d, const Frame *s)
{
#if defined(__CUDA_ARCH__)
    const uint4 *a = reinterpret_cast<const uint4 *>(s);
    uint4 *b = reinterpret_cast<uint4 *>(&d);
#pragma unroll
    for (int i = 0; i < FRAME_WORDS; i++)
        b[i] = __ldcg(a + i);
#else
    d = *s;
#endif
}
TB_D void frame_store_link(Frame *d, const Frame &s)
{
#if defined(__CUDA_ARCH__)
    const uint4 *a = reinterpret_cast<const uint4 *>(&s);
    uint4 *b = reinterpret_cast<uint4 *>(d);
#pragma unroll
    for (int i = 0; i < FRAME_WORDS; i++)
        __stcg(b + i, a[i]);
#else
    *d = s;
#endif
}
TB_D int64_t ts_load_link(const Frame *s)
{
#if defined(__CUDA_ARCH__)
    return __ldcg(&s->ts);
#else
    return s->ts;
#endif
}
TB_D int64_t tag_load(const int64_t *p)
{
#if defined(__CUDA_ARCH__)
    return __ldcg(p);
#else
    return *p;
#endif
}
TB_D void tag_store(int64_t *p, int64_t v)
{
#if defined(__CUDA_ARCH__)
    __stcg(p, v);
#else
    *p = v;
#endif
}

TB_D void ev_add(const Sim &s, int world, int i, unsigned long long n)
{
    if (!n)
        return;
#if defined(__CUDA_ARCH__)
    atomicAdd(&s.ev[i], n);
    atomicAdd(&s.ev_w[(size_t)world * EV_N + i], n);
#else
    s.ev[i] += n;
    s.ev_w[(size_t)world * EV_N + i] += n;
#endif
}

// link messages: slot `slot` of link `link`
TB_D size_t msg_index(const Sim &s, int64_t slot, int link) { return (size_t)(slot & (NB - 1)) * s.L + link; }
TB_D int msg_count(const Sim &s, int64_t slot, int link)
{
    int64_t v = tag_load(&s.msg_tag[msg_index(s, slot, link)]);
    return (v >> 16) == slot ? (int)(v & 0xFFFF) : 0;
}
TB_D const Frame *msg_frames(const Sim &s, int64_t slot, int link) { return s.msg + msg_index(s, slot, link) * MAX_TX; }

// The sending end of a point-to-point link for one slot: ns-3's RED queue disc over a one-packet
// device queue over the wire (reference: src/step.cuh:163-317). `ring` holds the frames that have
// not started, each stamped with its enqueue time; the wire is busy until `busy_until` with the
// frame that began at `began`, whose chain is *tx_chain. A frame begins at max(its enqueue time,
// busy_until); its transmission's copy, stamped with its arrival at the far end, goes to this
// slot's link message `msg` (at most MAX_TX; more is counted as an overflow).
// SHADOW: the frame enqueued last is also kept at *shadow (shared memory) with its ring index, so
// that a frame queued and started in the same slot is not read back from global memory.
template <bool SHADOW>
struct Transmitter
{
    Frame *ring;
    int cap, head, size;
    int64_t busy_until, began;
    Chain *tx_chain;
    int red_k, qcap;
    int64_t horizon;    // the slot's end: nothing begins at or after it
    int64_t kicked;     // the instant of a ScheduleNow'd event being handled (-1: none)
    int64_t idle_began; // the last start this slot on an idle wire (-1: none)
    Frame *msg;
    int n_out;
    unsigned drops, marks, ovf, offered;
    Frame *shadow;
    int shadow_at;
#ifdef TB_QTRACE
    const Sim *qs; // the trace's sink; the queue's ns-3 node and device
    int qnode, qdev;
#endif

    TB_D void open(Frame *ring_, int cap_, int head_, int size_, int64_t busy_until_, int64_t began_, Chain *tx_chain_, int red_k_,
                   int qcap_, int64_t horizon_, Frame *msg_)
    {
        ring = ring_;
        cap = cap_;
        head = head_;
        size = size_;
        busy_until = busy_until_;
        began = began_;
        tx_chain = tx_chain_;
        red_k = red_k_;
        qcap = qcap_;
        horizon = horizon_;
        kicked = idle_began = -1;
        msg = msg_;
        n_out = 0;
        drops = marks = ovf = offered = 0;
        shadow = nullptr;
        shadow_at = -1;
    }
    TB_D const Frame &at_head() const { return SHADOW && head == shadow_at ? *shadow : ring[head]; }

    // every waiting frame that begins by `until` (and before the horizon) goes on the wire; a frame
    // that found the wire busy begins at the previous one's TransmitComplete, whose chain is its
    // parent's; one that found it idle begins at its own enqueue, its chain unchanged
    TB_D void advance(int64_t until)
    {
        for (; size; size--)
        {
            const Frame &f = at_head();
            const int64_t t0 = f.ts > busy_until ? f.ts : busy_until;
            if (t0 > until || t0 >= horizon)
                return;
            if (n_out == MAX_TX)
            {
                ovf++;
                return;
            }
            const int64_t t1 = t0 + (int64_t)f.len * PS_PER_BYTE; // (its end, read before the stores below)
            const bool behind = busy_until >= f.ts && busy_until > began;
            Frame o;
            frame_copy(&o, &f);
            if (behind)
                chain_child(o.ch, *tx_chain, code_tc((int)((busy_until - began) / PS_PER_BYTE)));
            else
                idle_began = t0;
            *tx_chain = o.ch;
            began = t0;
            busy_until = t1;
            o.ts = t1 + PROP_PS;
            frame_store_link(&msg[n_out++], o);
            head = head + 1 == cap ? 0 : head + 1;
        }
    }

    // the frames RED counts at `now`: the waiting ones, less the one the device queue holds while
    // the wire is busy, once the Wake that refills it has run. The Wake is ScheduleNow'd when a
    // transmission begins, so it has run for one that began earlier; for one that began at this
    // instant only a ScheduleNow'd event sees it, after a start on an idle wire (a start at a
    // TransmitComplete comes after the arrivals that scheduled such events).
    TB_D int disc_backlog(int64_t now) const
    {
        if (!size || busy_until <= now)
            return size;
        const bool woken = began < now || (kicked == now && idle_began == now);
        return size - (woken ? 1 : 0);
    }

#ifdef TB_QTRACE
    TB_D void trace(const Frame &g, int backlog, int64_t now) const
    {
        if (!qs->qtrace || now >= qs->qtrace_until || now < qs->qtrace_from)
            return;
#if defined(__CUDA_ARCH__)
        const unsigned long long i = atomicAdd(qs->qtrace_cnt, 1ull);
#else
        const unsigned long long i = (*qs->qtrace_cnt)++;
#endif
        if (i >= qs->qtrace_n)
            return;
        QRec &r = qs->qtrace[i];
        const SndRec &S = qs->snd[g.flow];
        r.ts = now;
        r.node = qnode;
        r.dev = qdev;
        r.src = g.to_sender ? S.dst_local : S.src_local;
        r.dst = g.to_sender ? S.src_local : S.dst_local;
        r.sa = g.sa;
        r.len = g.len;
        r.qlen = (uint16_t)(backlog + 1);
        r.flags = g.flags;
    }
#endif

    // a frame offered at `now` (its ts becomes now): the wire first takes what begins by now; RED
    // with MinTh = MaxTh = K and weight 1 (no averaging) marks an ECT frame or drops another when
    // the backlog is at least K (and above 1); then the disc's limit drops. False: dropped.
    TB_D bool enqueue(Frame &g, int64_t now)
    {
        offered++;
        advance(now);
        const int backlog = disc_backlog(now);
        g.ts = now;
        if (backlog >= red_k && backlog > 1)
        {
            if (!(g.flags & F_ECT))
            {
                drops++;
                return false;
            }
            g.flags |= F_CE;
            marks++;
        }
        if (backlog >= qcap)
        {
            drops++;
            return false;
        }
#ifdef TB_QTRACE
        trace(g, backlog, now);
#endif
        if (size == cap)
        {
            ovf++;
            return false;
        }
        const int at = head + size < cap ? head + size : head + size - cap;
        frame_copy(&ring[at], &g);
        if (SHADOW)
        {
            *shadow = g;
            shadow_at = at;
        }
        size++;
        return true;
    }
};
using Egress = Transmitter<false>;
using PortEgress = Transmitter<true>;

} // namespace tb
