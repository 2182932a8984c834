// twins-b200: one slot of a host and of a switch.
//   host_step   (reference: src/step.cuh:2250-2528) one thread per host: every event of the host
//               in [t us, t+1 us) in ns-3's order: arrivals, timers, application starts
//   switch_step (reference: src/step.cuh:2530-2886) one warp per switch, one lane per port:
//               ingress windows -> routes (per-flow ECMP or MRG32k3a spraying) -> counting sort to
//               egress ports -> per-egress ordering by (time, ns-3 order) -> RED enqueue -> starts
#pragma once
#include "tb_tcp.cuh"

namespace tb
{

// the chain of a timer (due_chain, step.cuh:2241-2247)
TB_D const Chain &due_chain(const Sim &s, const Due &d)
{
    switch (d.kind)
    {
    case 1:
    case 3:
    case 4:
        return s.rcv[d.flow].dchain;
    case 5:
        return s.rcv[d.flow].fchain;
    case 2:
        return s.snd[d.flow].st == S_EST ? s.snd[d.flow].schain : s.snd[d.flow].rchain;
    default:
        return s.snd[d.flow].rchain;
    }
}

// a receiver that can arm no timer any more: all its timers idle and everything received (or,
// with FIN, the connection closed)
TB_D bool rcv_idle_for_good(const RcvRec &R)
{
    if (R.delack_at >= 0 || R.syn_at >= 0 || R.last_at >= 0 || R.frx_at >= 0)
        return false;
    if (R.fin_on)
        return R.st == R_CLOSED;
    return R.est && R.rcv_nxt >= R.bytes;
}

// One slot of host h. Returns true if it sent or holds frames; *wake: the next slot it must run.
// t: the world's own slot (time); gt: the launch's slot, which indexes the link messages (equal
// in a batch; a world that joins a running launch starts its own time at a later launch slot).
// `stage`: the host's link messages of slots gt-2 and gt-1 copied to shared memory by its warp
// (msg[gt-2] then msg[gt-1], n2 and n1 frames as their tags count), or null to read them in place
// (n2, n1 < 0: read the tags).
// prune_later: the active lists are left unpruned and *wake counts only the host's queue and its
// next application start; the caller prunes them (prune_lists_warp) and lowers the wake-up to the
// earliest timer of the connections that stay. `due`: the timers due in the slot, already collected
// in this function's scan order (the first DUE_CAP of them; due_ovf more were left out), or null
// to scan the active lists here.
TB_D bool host_step(const Sim &s, int h, int64_t t, int64_t gt, int64_t *wake, unsigned *ties_out, unsigned *done_out,
                    const Frame *stage = nullptr, int n2 = -1, int n1 = -1, bool prune_later = false, const Due *due = nullptr,
                    int due_n = 0, int due_ovf = 0)
{
    const int64_t S0 = t * SLOT_PS, E0 = S0 + SLOT_PS;
    TB_PHASE_START
    HostRec &hr = s.hosts[h];
    const int link = hr.in_link;
    const Frame *m2 = nullptr, *m1 = nullptr;
    int i2 = 0, i1 = 0;
    auto ts_at = [&](const Frame *m, int j) { return stage ? m[j].ts : ts_load_link(&m[j]); };
    auto frame_at = [&](Frame &d, const Frame *m, int j) {
        if (stage)
            d = m[j];
        else
            frame_load_link(d, &m[j]);
    };
    if (n2 < 0)
        n2 = gt >= 2 ? msg_count(s, gt - 2, link) : 0;
    if (n1 < 0)
        n1 = gt >= 1 ? msg_count(s, gt - 1, link) : 0;
    if (n2 > 0)
    {
        m2 = stage ? stage : msg_frames(s, gt - 2, link);
        while (i2 < n2 && ts_at(m2, i2) < S0)
            i2++;
    }
    if (n1 > 0)
        m1 = stage ? stage + n2 : msg_frames(s, gt - 1, link);
    bool input = i2 < n2 || (n1 > 0 && ts_at(m1, 0) < E0);
    if (!input && t < hr.wake && hr.q_size == 0)
    {
        *wake = hr.wake;
        return false;
    }
    const WorldDesc &wd = s.worlds[hr.world];
    HostCtx c;
    c.s = &s;
    c.wd = &wd;
    c.h = h;
    c.dctcp = wd.cc == CC_DCTCP;
    c.cubic = wd.cc == CC_CUBIC;
    c.slot_end = E0;
    c.retx = c.rtos = c.ovf = c.done = 0;
    c.pkts = c.snd_pkts = 0;
    Egress &nic = c.nic;
    nic.open(s.host_ring + (size_t)h * s.ring, s.ring, hr.q_head, hr.q_size, hr.link_free, hr.last_start, &hr.last, wd.red_k, wd.qcap, E0,
             s.msg + msg_index(s, gt, h) * MAX_TX);
#ifdef TB_QTRACE
    nic.qs = &s;
    nic.qnode = hr.local;
    nic.qdev = 1;
#endif
    unsigned ties = 0;

    TB_PHASE(0)
    // timers due in this slot (new timers lie >= 10 us ahead, except the 1 ps Send deferral,
    // which timer_in_slot adds), by time
    int *act_snd = s.act_snd + (size_t)h * s.act_cap, *act_rcv = s.act_rcv + (size_t)h * s.act_cap;
    const int ns = hr.n_snd, nr = hr.n_rcv;
    c.nd = 0;
    c.di = 0;
    if (due)
    {
        for (int i = 0; i < due_n; i++)
            c.due[i] = due[i];
        c.nd = due_n;
        c.ovf += due_ovf;
    }
    for (int i = 0; i < (due ? 0 : ns); i++)
    {
        int f = act_snd[i];
        const SndRec &S = s.snd[f];
        int64_t a = S.rto_at, b = S.syn_at;
        if (a >= 0 && a < E0)
        {
            if (c.nd < DUE_CAP)
                c.due[c.nd++] = {a, f, 0};
            else
                c.ovf++;
        }
        if (b >= 0 && b < E0)
        {
            if (c.nd < DUE_CAP)
                c.due[c.nd++] = {b, f, 2};
            else
                c.ovf++;
        }
    }
    for (int i = 0; i < (due ? 0 : nr); i++)
    {
        int f = act_rcv[i];
        const RcvRec &R = s.rcv[f];
        int64_t v[4] = {R.delack_at, R.syn_at, R.last_at, R.frx_at};
        const int kinds[4] = {1, 3, 4, 5};
        for (int j = 0; j < 4; j++)
            if (v[j] >= 0 && v[j] < E0)
            {
                if (c.nd < DUE_CAP)
                    c.due[c.nd++] = {v[j], f, kinds[j]};
                else
                    c.ovf++;
            }
    }
    for (int i = 1; i < c.nd; i++)
    {
        Due x = c.due[i];
        int j = i - 1;
        while (j >= 0 && c.due[j].at > x.at)
        {
            c.due[j + 1] = c.due[j];
            j--;
        }
        c.due[j + 1] = x;
    }
    TB_PHASE(1)
    int pn = hr.pend_next;
    const int pe = hr.pend_end;
    Frame p;
    bool have_p = false; // p holds the next arrival
    for (;;)
    {
        int64_t tr = INT64_MAX, td = INT64_MAX, tp = INT64_MAX;
        if (!have_p)
        {
            if (i2 < n2)
            {
                frame_at(p, m2, i2);
                have_p = true;
            }
            else if (i1 < n1 && ts_at(m1, i1) < E0)
            {
                frame_at(p, m1, i1);
                have_p = true;
            }
        }
        if (have_p)
            tr = p.ts;
        if (c.di < c.nd)
            td = c.due[c.di].at;
        int pm = -1;
        if (pn < pe)
        {
            pm = s.pend_msg[pn];
            int64_t st = s.msgs[pm].start;
            if (st < E0)
                tp = st;
        }
        int64_t now = tr < td ? tr : td;
        now = now < tp ? now : tp;
        if (now == INT64_MAX)
            break;
        if (now < S0)
            now = S0;
        TB_PHASE(2)
        nic.advance(now);
        TB_PHASE(8)
        if (now == tp)
        {
            pn++;
            app_event(c, hr, act_snd, pm, now);
            TB_PHASE(10)
            continue;
        }
        bool timer = now == td;
        if (timer && now == tr)
        {
            // a timer and an arrival at the same instant: the one scheduled first
            Chain arr;
            chain_child(arr, p.ch, code_arrival(p.len));
            int r = chain_cmp(due_chain(s, c.due[c.di]), arr);
            if (r == 0)
                ties++;
            timer = r <= 0; // (undecided: the timer)
        }
        if (timer)
        {
            const Due d = c.due[c.di++];
            c.ech = due_chain(s, d);
            timer_event(c, d, now);
            TB_PHASE(10)
            continue;
        }
        // the arrival
        if (i2 < n2)
            i2++;
        else
            i1++;
        have_p = false;
        c.pkts++;
        c.snd_pkts += p.to_sender;
        chain_child(c.ech, p.ch, code_arrival(p.len));
        on_frame(c, hr, p, now);
        TB_PHASE(9)
    }
    TB_PHASE(2)
    nic.advance(E0 - 1);
    tag_store(&s.msg_tag[msg_index(s, gt, h)], (int64_t)gt << 16 | nic.n_out);
    hr.q_head = nic.head;
    hr.q_size = nic.size;
    hr.link_free = nic.busy_until;
    hr.last_start = nic.began;
    hr.pend_next = pn;

    TB_PHASE(3)
    // drop finished connections from the active lists; the next wake-up
    int64_t next = INT64_MAX;
    if (!prune_later)
    {
        int k = 0, n = hr.n_snd;
        for (int i = 0; i < n; i++)
        {
            int f = act_snd[i];
            const SndRec &S = s.snd[f];
            if (S.st == S_DONE)
                continue;
            act_snd[k++] = f;
            if (S.rto_at >= 0 && S.rto_at < next)
                next = S.rto_at;
            if (S.syn_at >= 0 && S.syn_at < next)
                next = S.syn_at;
        }
        hr.n_snd = k;
    }
    if (!prune_later)
    {
        int k = 0, n = hr.n_rcv;
        for (int i = 0; i < n; i++)
        {
            int f = act_rcv[i];
            const RcvRec &R = s.rcv[f];
            if (rcv_idle_for_good(R))
                continue;
            act_rcv[k++] = f;
            int64_t v[4] = {R.delack_at, R.syn_at, R.last_at, R.frx_at};
            for (int j = 0; j < 4; j++)
                if (v[j] >= 0 && v[j] < next)
                    next = v[j];
        }
        hr.n_rcv = k;
    }
    if (pn < pe)
    {
        int64_t st = s.msgs[s.pend_msg[pn]].start;
        if (st < next)
            next = st;
    }
    hr.wake = nic.size > 0 ? t + 1 : (next == INT64_MAX ? INT64_MAX : next / SLOT_PS);
    *wake = hr.wake;
    TB_PHASE(4)
    // counters
    ev_add(s, hr.world, EV_DROPS, nic.drops);
    ev_add(s, hr.world, EV_MARKS, nic.marks);
    ev_add(s, hr.world, EV_RETX, c.retx);
    ev_add(s, hr.world, EV_RTO, c.rtos);
    ev_add(s, hr.world, EV_HOST_PKT, c.pkts);
    ev_add(s, hr.world, EV_HOST_SND, c.snd_pkts);
    ev_add(s, hr.world, EV_HOST_FRAMES, nic.offered);
    ev_add(s, hr.world, EV_OVF_RING, c.ovf);
    ev_add(s, hr.world, EV_OVF_TX, nic.ovf);
    ev_add(s, hr.world, EV_TIES, ties);
    *ties_out += ties;
    *done_out += c.done;
    TB_PHASE(5)
    return nic.n_out > 0 || nic.size > 0;
}

// ------------------------------------------------------------------ switches
TB_D int epoch_of(const WorldDesc &wd, int64_t ts)
{
    int e = 0;
    while (e < wd.n_fail && ts >= wd.fail_t[e])
        e++;
    return e;
}
// the egress port at switch sw (world-local) towards host dst (world-local); `up` indexes the
// equal-cost routes (reference: src/step.cuh:2554-2591)
TB_D int route_up(const WorldDesc &wd, int sw, int dst, int up, int ep)
{
    if (wd.kind == TOPO_GRAPH)
    {
        int e = wd.host_sw[dst];
        if (e == sw)
            return wd.host_port[dst];
        size_t r = ((size_t)ep * wd.S1 + sw) * wd.S1 + e;
        return wd.rt_ports[wd.rt_off[r] + up];
    }
    if (wd.kind == TOPO_LEAFSPINE)
    {
        if (sw < wd.leaves)
            return dst / wd.hpl == sw ? dst % wd.hpl : wd.hpl + up;
        return dst / wd.hpl;
    }
    const int k = wd.k, hk = wd.hk, E = k * hk;
    int dst_pod = dst / (hk * hk), dst_edge = (dst / hk) % hk;
    if (sw < E)
        return (dst_pod == sw / hk && dst_edge == sw % hk) ? dst % hk : hk + up;
    if (sw < 2 * E)
        return dst_pod == (sw - E) / hk ? dst_edge : hk + up;
    return dst_pod;
}
TB_D int route(const Sim &s, const WorldDesc &wd, int sw, const Frame &p, int ep)
{
    if (wd.kind == TOPO_GRAPH)
    {
        int e = wd.host_sw[p.dst];
        if (e == sw)
            return wd.host_port[p.dst];
        // the flow hash modulo the routes at this switch
        const SndRec &S = s.snd[p.flow];
        uint32_t hsh = p.to_sender ? S.hash_ack : S.hash_data;
        return route_up(wd, sw, p.dst, (int)(hsh % wd.rt_n[((size_t)ep * wd.S1 + sw) * wd.S1 + e]), ep);
    }
    return route_up(wd, sw, p.dst, p.up, ep);
}
TB_D bool port_down(const WorldDesc &wd, int sw, int q, int ep)
{
    return wd.n_fail && wd.port_dn[((size_t)ep * wd.S1 + sw) * wd.k + q];
}
// equal-cost routes Ipv4GlobalRouting finds from sw towards dst (0: the host is attached)
TB_D int routes_to(const WorldDesc &wd, int sw, int dst, int ep)
{
    if (wd.kind == TOPO_GRAPH)
        return wd.host_sw[dst] == sw ? 0 : wd.rt_n[((size_t)ep * wd.S1 + sw) * wd.S1 + wd.host_sw[dst]];
    if (wd.kind == TOPO_LEAFSPINE)
        return sw < wd.leaves ? (dst / wd.hpl == sw ? 0 : wd.ecmp_n) : 1;
    const int hk = wd.hk, E = wd.k * hk;
    int dst_pod = dst / (hk * hk), dst_edge = (dst / hk) % hk;
    if (sw < E)
        return dst_pod == sw / hk && dst_edge == sw % hk ? 0 : wd.ecmp_n;
    if (sw < 2 * E)
        return dst_pod == (sw - E) / hk ? 1 : wd.ecmp_n;
    return 1;
}

// simultaneous arrivals at a switch, as ns-3 orders their Receive events: the longer frame
// started earlier upstream; else the chains of the upstream starts; else the lower connection id
// (a guess, counted) (frame_before, step.cuh:2693-2705)
TB_D bool frame_before(const Frame &a, const Frame &b, unsigned &ties)
{
    if (a.len != b.len)
        return a.len > b.len;
    int c = chain_cmp(a.ch, b.ch);
    if (c == 0)
        ties++;
    return c != 0 ? c < 0 : a.flow < b.flow;
}

} // namespace tb
