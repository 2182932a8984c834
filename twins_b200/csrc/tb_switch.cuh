// twins-b200: one slot of one switch as phases of its warp, one lane per port (k <= 32).
// The phases are separated by warp barriers on the device (switch_step in tb_kernel.cu).
// Reference: src/step.cuh:2748-2886 (switch_step), :2709-2745 (spray_draws).
#pragma once
#include "tb_slot.cuh"

namespace tb
{

struct SwCtx
{
    const Sim *s;
    const WorldDesc *wd;
    const SwRec *sr;
    int sw;        // global switch id
    PortRec *ports; // the switch's ports
    size_t scratch; // its region in sw_ts / sw_ref / sw_up
    int64_t t;
    bool spray;
};

TB_D int sw_egress_of(const SwCtx &x, const SwShared &sh, int q, int j, const Frame *p)
{
    const WorldDesc &wd = *x.wd;
    int ep = wd.n_fail ? epoch_of(wd, ts_load_link(p)) : 0;
    if (port_down(wd, x.sr->local, q, ep))
        return -1; // dropped on arrival at a down interface
    Frame f;
    frame_load_link(f, p);
    if (x.spray)
        return route_up(wd, x.sr->local, f.dst, x.s->sw_up[x.scratch + (size_t)q * 2 * MAX_TX + j], ep);
    return route(*x.s, wd, x.sr->local, f, ep);
}

// phase 1 (lane q): the ingress window; clear the row
TB_D int sw_phase_window(const SwCtx &x, SwShared &sh, int q)
{
    Input in = input_window(*x.s, x.ports[q].in_link, x.t);
    sh.win[q][0] = in.i2;
    sh.win[q][1] = in.n2;
    sh.win[q][2] = in.n1;
    for (int i = 0; i <= x.sr->k; i++)
        sh.rows[q][i] = 0;
    return in.count();
}

// phase 2 (one lane): per-packet ECMP draws, one per forwarded packet in the order the packets
// arrive at the node (all ports merged), from the switch's MRG32k3a stream
TB_D void sw_phase_spray(const SwCtx &x, const SwShared &sh, unsigned &ties)
{
    const int k = x.sr->k;
    int pos[32];
    for (int q = 0; q < k; q++)
        pos[q] = 0;
    Rng st = x.s->sw_rng[x.sw];
    const WorldDesc &wd = *x.wd;
    for (;;)
    {
        int best = -1;
        Frame bf, f;
        for (int q = 0; q < k; q++)
        {
            Input in = input_cached(*x.s, sh, x.ports, q, x.t);
            if (pos[q] >= in.count())
                continue;
            frame_load_link(f, in.at(pos[q]));
            if (best < 0 || f.ts < bf.ts || (f.ts == bf.ts && frame_before(f, bf, ties)))
            {
                best = q;
                bf = f;
            }
        }
        if (best < 0)
            break;
        int ep = wd.n_fail ? epoch_of(wd, bf.ts) : 0;
        if (!port_down(wd, x.sr->local, best, ep))
        {
            int nr = routes_to(wd, x.sr->local, bf.dst, ep);
            x.s->sw_up[x.scratch + (size_t)best * 2 * MAX_TX + pos[best]] = (uint8_t)(nr ? rand_int(st, (uint32_t)nr) : 0);
        }
        pos[best]++;
    }
    x.s->sw_rng[x.sw] = st;
}

// phase 3 (lane q): count arrivals per egress port; returns the drops at a down interface
TB_D unsigned sw_phase_count(const SwCtx &x, SwShared &sh, int q)
{
    Input in = input_cached(*x.s, sh, x.ports, q, x.t);
    unsigned dropped = 0;
    int n = in.count();
    for (int j = 0; j < n; j++)
    {
        int e = sw_egress_of(x, sh, q, j, in.at(j));
        if (e >= 0)
            sh.rows[q][e]++;
        else
            dropped++;
    }
    return dropped;
}

// phase 4 (lane e): offsets of each ingress port's arrivals within egress e
TB_D void sw_phase_offsets(const SwCtx &x, SwShared &sh, int e)
{
    int off = 0;
    for (int j = 0; j < x.sr->k; j++)
    {
        int c = sh.rows[j][e];
        sh.rows[j][e] = off;
        off += c;
    }
    sh.cnt[e] = off;
}

// phase 5 (lane e): egress e's region in the scratch
TB_D void sw_phase_base(const SwCtx &x, SwShared &sh, int e)
{
    int b = 0;
    for (int j = 0; j < e; j++)
        b += sh.cnt[j];
    sh.base[e] = b;
}

// phase 6 (lane q): scatter (time, source) of each arrival to its egress region
TB_D void sw_phase_scatter(const SwCtx &x, SwShared &sh, int q)
{
    Input in = input_cached(*x.s, sh, x.ports, q, x.t);
    int n = in.count();
    for (int j = 0; j < n; j++)
    {
        const Frame *p = in.at(j);
        int e = sw_egress_of(x, sh, q, j, p);
        if (e < 0)
            continue;
        int at = sh.base[e] + sh.rows[q][e]++;
        x.s->sw_ts[x.scratch + at] = ts_load_link(p);
        x.s->sw_ref[x.scratch + at] = (uint32_t)(q << 16 | j);
    }
}

// phase 7 (lane e): egress e's arrivals in time order (ties: ns-3's order, insertion sort in
// ingress order), each enqueued (RED) with its arrival event's chain; then the starts of the
// slot. Returns true if the port sent or holds frames.
TB_D bool sw_phase_egress(const SwCtx &x, const SwShared &sh, int e, unsigned &ties, unsigned &drops, unsigned &marks,
                          unsigned &ovf)
{
    const Sim &s = *x.s;
    const int n = sh.cnt[e];
    int64_t *ts = s.sw_ts + x.scratch + sh.base[e];
    uint32_t *ref = s.sw_ref + x.scratch + sh.base[e];
    auto frame_at = [&](uint32_t r) -> const Frame * {
        Input src = input_cached(s, sh, x.ports, (int)(r >> 16), x.t);
        return src.at((int)(r & 0xFFFF));
    };
    for (int i = 1; i < n; i++)
    {
        int64_t tx = ts[i];
        uint32_t r = ref[i];
        int j = i - 1;
        while (j >= 0)
        {
            if (ts[j] < tx)
                break;
            if (ts[j] == tx)
            {
                Frame a, b;
                frame_load_link(a, frame_at(r));
                frame_load_link(b, frame_at(ref[j]));
                if (!frame_before(a, b, ties))
                    break;
            }
            ts[j + 1] = ts[j];
            ref[j + 1] = ref[j];
            j--;
        }
        ts[j + 1] = tx;
        ref[j + 1] = r;
    }
    PortRec &pr = x.ports[e];
    const int port = x.sr->port0 + e;
    Egress eg;
    eg.ring = s.port_ring + (size_t)port * s.ring;
    eg.cap = s.ring;
    eg.head = pr.q_head;
    eg.size = pr.q_size;
    eg.link_free = pr.link_free;
    eg.last_start = pr.last_start;
    eg.last = &pr.last;
    eg.red_k = pr.red_k;
    eg.qcap = pr.qcap;
    eg.woke = -1;
    eg.idle_start = -1;
    eg.slot_end = (x.t + 1) * SLOT_PS;
    const int out_link = s.H + port;
    eg.out = s.msg + msg_index(s, x.t, out_link) * MAX_TX;
    eg.sent = 0;
    eg.drops = eg.marks = eg.ovf = eg.emitted = 0;
    for (int i = 0; i < n; i++)
    {
        Frame p;
        frame_load_link(p, frame_at(ref[i]));
        chain_child(p.ch, p.ch, code_arrival(p.len)); // queued: the arrival event's chain
        eg.enqueue(p, p.ts);
    }
    eg.advance(eg.slot_end - 1);
    tag_store(&s.msg_tag[msg_index(s, x.t, out_link)], (int64_t)x.t << 16 | eg.sent);
    pr.q_head = eg.head;
    pr.q_size = eg.size;
    pr.link_free = eg.link_free;
    pr.last_start = eg.last_start;
    drops += eg.drops;
    marks += eg.marks;
    ovf += eg.ovf;
    return eg.sent > 0 || eg.size > 0;
}

} // namespace tb
