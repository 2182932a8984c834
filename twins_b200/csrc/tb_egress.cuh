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

// The egress port's working copy for one slot (reference: src/step.cuh:163-317, Fifo).
struct Egress
{
    Frame *ring;
    int cap, head, size;
    int64_t link_free, last_start;
    Chain *last; // persistent: the chain of the transmission in progress
    int red_k, qcap;
    int64_t woke, idle_start, slot_end;
    Frame *out; // this slot's link message
    int sent;
    unsigned drops, marks, ovf, emitted;
#ifdef TB_QTRACE
    const Sim *qs; // the trace's sink; the queue's ns-3 node and device
    int qnode, qdev;
#endif

    // start every frame whose transmission begins by `until` and within this slot
    TB_D void advance(int64_t until)
    {
        while (size > 0)
        {
            Frame *f = &ring[head];
            int64_t start = f->ts > link_free ? f->ts : link_free;
            if (start > until || start >= slot_end)
                return;
            if (sent >= MAX_TX)
            {
                ovf++;
                return;
            }
            int64_t end = start + (int64_t)f->len * PS_PER_BYTE;
            Frame o;
            frame_copy(&o, f);
            // its parent event: the previous frame's TransmitComplete, unless the link was idle
            if (f->ts <= link_free && link_free > last_start)
                chain_child(o.ch, *last, code_tc((int)((link_free - last_start) / PS_PER_BYTE)));
            else
                idle_start = start;
            *last = o.ch;
            last_start = start;
            o.ts = end + PROP_PS;
            frame_store_link(&out[sent], o);
            sent++;
            link_free = end;
            head = head + 1 == cap ? 0 : head + 1;
            size--;
        }
    }

    // RED with MinTh = MaxTh = K and QW = 1 on the queue disc's length, which excludes the
    // device queue's packet once ns-3's Wake (ScheduleNow) has refilled it; then the limit
    TB_D bool enqueue(Frame &g, int64_t now)
    {
        emitted++;
        advance(now);
        bool refilled = last_start < now || (woke == now && idle_start == now);
        int nq = (size > 0 && link_free > now && refilled) ? size - 1 : size;
        g.ts = now;
        if (nq >= red_k && nq > 1)
        {
            if (g.flags & F_ECT)
            {
                g.flags |= F_CE;
                marks++;
            }
            else
            {
                drops++;
                return false;
            }
        }
        if (nq >= qcap)
        {
            drops++;
            return false;
        }
#ifdef TB_QTRACE
        if (qs->qtrace && now < qs->qtrace_until && now >= qs->qtrace_from)
        {
#if defined(__CUDA_ARCH__)
            const unsigned long long i = atomicAdd(qs->qtrace_cnt, 1ull);
#else
            const unsigned long long i = (*qs->qtrace_cnt)++;
#endif
            if (i < qs->qtrace_n)
            {
                QRec &r = qs->qtrace[i];
                const SndRec &S = qs->snd[g.flow];
                r.ts = now;
                r.node = qnode;
                r.dev = qdev;
                r.src = g.to_sender ? S.dst_local : S.src_local;
                r.dst = g.to_sender ? S.src_local : S.dst_local;
                r.sa = g.sa;
                r.len = g.len;
                r.qlen = (uint16_t)(nq + 1);
                r.flags = g.flags;
            }
        }
#endif
        if (size >= cap)
        {
            ovf++;
            return false;
        }
        int at = head + size;
        if (at >= cap)
            at -= cap;
        frame_copy(&ring[at], &g);
        size++;
        return true;
    }
};

// A switch port's working copy for one slot, as Egress, with the chain of the transmission in
// progress and the frame last enqueued kept in the warp's shared scratch for the slot (the caller
// loads the chain and stores it back), so that a started frame does not read back from L2 what
// the step before had just written. (A separate kernel instantiation uses it: the plain Egress
// keeps the other one's code as it is.)
struct PortEgress
{
    Frame *ring;
    int cap, head, size;
    int64_t link_free, last_start;
    Chain *last; // the chain of the transmission in progress: the slot's copy in shared memory
    Frame *tailp; // the frame last enqueued (ring index tail_at; -1: none), in shared memory
    int tail_at;
    int red_k, qcap;
    int64_t woke, idle_start, slot_end;
    Frame *out; // this slot's link message
    int sent;
    unsigned drops, marks, ovf, emitted;
#ifdef TB_QTRACE
    const Sim *qs; // the trace's sink; the queue's ns-3 node and device
    int qnode, qdev;
#endif

    // start every frame whose transmission begins by `until` and within this slot
    TB_D void advance(int64_t until)
    {
        while (size > 0)
        {
            const Frame *f = head == tail_at ? tailp : &ring[head];
            int64_t start = f->ts > link_free ? f->ts : link_free;
            if (start > until || start >= slot_end)
                return;
            if (sent >= MAX_TX)
            {
                ovf++;
                return;
            }
            int64_t end = start + (int64_t)f->len * PS_PER_BYTE;
            Frame o;
            frame_copy(&o, f);
            // its parent event: the previous frame's TransmitComplete, unless the link was idle
            if (f->ts <= link_free && link_free > last_start)
                chain_child(o.ch, *last, code_tc((int)((link_free - last_start) / PS_PER_BYTE)));
            else
                idle_start = start;
            *last = o.ch;
            last_start = start;
            o.ts = end + PROP_PS;
            frame_store_link(&out[sent], o);
            sent++;
            link_free = end;
            head = head + 1 == cap ? 0 : head + 1;
            size--;
        }
    }

    // RED with MinTh = MaxTh = K and QW = 1 on the queue disc's length, which excludes the
    // device queue's packet once ns-3's Wake (ScheduleNow) has refilled it; then the limit
    TB_D bool enqueue(Frame &g, int64_t now)
    {
        emitted++;
        advance(now);
        bool refilled = last_start < now || (woke == now && idle_start == now);
        int nq = (size > 0 && link_free > now && refilled) ? size - 1 : size;
        g.ts = now;
        if (nq >= red_k && nq > 1)
        {
            if (g.flags & F_ECT)
            {
                g.flags |= F_CE;
                marks++;
            }
            else
            {
                drops++;
                return false;
            }
        }
        if (nq >= qcap)
        {
            drops++;
            return false;
        }
#ifdef TB_QTRACE
        if (qs->qtrace && now < qs->qtrace_until && now >= qs->qtrace_from)
        {
#if defined(__CUDA_ARCH__)
            const unsigned long long i = atomicAdd(qs->qtrace_cnt, 1ull);
#else
            const unsigned long long i = (*qs->qtrace_cnt)++;
#endif
            if (i < qs->qtrace_n)
            {
                QRec &r = qs->qtrace[i];
                const SndRec &S = qs->snd[g.flow];
                r.ts = now;
                r.node = qnode;
                r.dev = qdev;
                r.src = g.to_sender ? S.dst_local : S.src_local;
                r.dst = g.to_sender ? S.src_local : S.dst_local;
                r.sa = g.sa;
                r.len = g.len;
                r.qlen = (uint16_t)(nq + 1);
                r.flags = g.flags;
            }
        }
#endif
        if (size >= cap)
        {
            ovf++;
            return false;
        }
        int at = head + size;
        if (at >= cap)
            at -= cap;
        frame_copy(&ring[at], &g);
        *tailp = g;
        tail_at = at;
        size++;
        return true;
    }
};

} // namespace tb
