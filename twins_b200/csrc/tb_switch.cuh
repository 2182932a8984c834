// twins-b200: one slot of one switch as phases of its warp (k <= 32 ports).
// Reference: src/step.cuh:2748-2886 (switch_step), :2709-2745 (spray_draws).
//
// The warp first copies every frame of the slot's ingress link messages into shared memory in
// one cooperative pass (all lanes, 16-byte loads from L2), so that the serial parts (the merged
// arrival order of per-packet spraying, each egress port's ordering and enqueues) read shared
// memory instead of making one dependent L2 round trip per frame. A slot whose messages exceed
// the staging area reads them in place (the same phases, through L2).
#pragma once
#include "tb_slot.cuh"

#include <type_traits>

namespace tb
{

// per-warp shared scratch of a switch (also a host unit's staging area). The staging arrays
// follow the header in the warp's part of the block's dynamic shared memory; their capacity
// (`cap` frames) is chosen per launch.
struct SwShared
{
    int rows[32][33];       // [ingress][egress] counts, then offsets
    int base[32], cnt[32];
    int win[32][3];         // each ingress port's window in its messages: (i2, n2, n1)
    int raw2[32], raw1[32]; // frames in the port's msg[t-2] / msg[t-1]
    int off2[32], off1[32]; // where they start in `fr` (staged)
    int staged, total;
    int cap;
    // the arrays after this header, addressed from the scratch itself (so that the compiler keeps
    // them in the shared address space): the staged frames [cap], then each egress region's
    // arrival times [cap] and sources [cap] (staged slots)
    TB_D unsigned char *bytes() { return reinterpret_cast<unsigned char *>(this); }
    TB_D const unsigned char *bytes() const { return reinterpret_cast<const unsigned char *>(this); }
    TB_D Frame *fr() { return reinterpret_cast<Frame *>(bytes() + header()); }
    TB_D const Frame *fr() const { return reinterpret_cast<const Frame *>(bytes() + header()); }
    TB_D int64_t *ets() { return reinterpret_cast<int64_t *>(bytes() + header() + (size_t)cap * sizeof(Frame)); }
    TB_D uint32_t *eref() { return reinterpret_cast<uint32_t *>(bytes() + header() + (size_t)cap * (sizeof(Frame) + 8)); }
    // (port-local egress) each port's frame last enqueued [32] and transmission chain [32]
    TB_D Frame *eg_tail() { return reinterpret_cast<Frame *>(bytes() + ports_at(cap)); }
    TB_D Chain *eg_last() { return reinterpret_cast<Chain *>(bytes() + ports_at(cap) + 32 * sizeof(Frame)); }
    static TB_HDI size_t header();
    static TB_HDI size_t ports_at(int cap);
};

TB_HDI size_t SwShared::header() { return (sizeof(SwShared) + 15) & ~(size_t)15; }
TB_HDI size_t SwShared::ports_at(int cap) { return (header() + (size_t)cap * (sizeof(Frame) + 8 + 4) + 15) & ~(size_t)15; }
// bytes of one warp's scratch with `cap` staged frames (16-byte multiple), and the ports' slot
// copies of the port-local egress
TB_HDI size_t sw_shared_bytes(int cap, bool port_local = false)
{
    return SwShared::ports_at(cap) + (port_local ? (32 * (sizeof(Frame) + sizeof(Chain)) + 15) & ~(size_t)15 : 0);
}
// a warp's scratch at `p` (every lane may call it: the same value is written)
TB_D SwShared *sw_shared_at(unsigned char *p, int cap)
{
    SwShared *sh = reinterpret_cast<SwShared *>(p);
    sh->cap = cap;
    return sh;
}

// ingress window of a port: the tail of msg[t-2] from S0 on, the head of msg[t-1] before E0;
// frames in shared memory (staged) or in the link messages
struct Input
{
    const Frame *m2, *m1;
    int i2, n2, n1;
    bool smem;
    TB_D int count() const { return (n2 - i2) + n1; }
    TB_D const Frame *at(int j) const { return j < n2 - i2 ? &m2[i2 + j] : &m1[j - (n2 - i2)]; }
    TB_D void load(Frame &f, int j) const
    {
        if (smem)
            f = *at(j);
        else
            frame_load_link(f, at(j));
    }
    TB_D int64_t ts(int j) const { return smem ? at(j)->ts : ts_load_link(at(j)); }
};

struct SwCtx
{
    const Sim *s;
    const WorldDesc *wd;
    const SwRec *sr;
    int sw;          // global switch id
    PortRec *ports;  // the switch's ports
    size_t scratch;  // its region in sw_ts / sw_ref / sw_up
    int64_t t;       // the world's own slot (time)
    int64_t gt;      // the launch's slot (indexes the link messages)
    bool spray;
};

TB_D Input input_of(const SwCtx &x, const SwShared &sh, int q)
{
    Input in;
    in.i2 = sh.win[q][0];
    in.n2 = sh.win[q][1];
    in.n1 = sh.win[q][2];
    in.smem = sh.staged != 0;
    if (in.smem)
    {
        in.m2 = &sh.fr()[sh.off2[q]];
        in.m1 = &sh.fr()[sh.off1[q]];
        return in;
    }
    int link = x.ports[q].in_link;
    if (link < 0)
        link = 0; // (an unused port's window is empty; any link gives valid pointers)
    in.m2 = x.gt >= 2 ? msg_frames(*x.s, x.gt - 2, link) : nullptr;
    in.m1 = x.gt >= 1 ? msg_frames(*x.s, x.gt - 1, link) : nullptr;
    return in;
}

// phase 1a (lane q < k): the port's message sizes; clear its row
TB_D void sw_phase_sizes(const SwCtx &x, SwShared &sh, int q)
{
    const Sim &s = *x.s;
    int link = x.ports[q].in_link;
    sh.raw2[q] = link >= 0 && x.gt >= 2 ? msg_count(s, x.gt - 2, link) : 0;
    sh.raw1[q] = link >= 0 && x.gt >= 1 ? msg_count(s, x.gt - 1, link) : 0;
    for (int i = 0; i <= x.sr->k; i++)
        sh.rows[q][i] = 0;
}

// phase 1b (lane 0): staging offsets
TB_D void sw_phase_layout(const SwCtx &x, SwShared &sh)
{
    int off = 0;
    for (int q = 0; q < x.sr->k; q++)
    {
        sh.off2[q] = off;
        off += sh.raw2[q];
        sh.off1[q] = off;
        off += sh.raw1[q];
    }
    sh.staged = off <= sh.cap;
    sh.total = off;
}

// phase 1c (every lane of the warp): copy the messages into shared memory
TB_D void sw_phase_copy(const SwCtx &x, SwShared &sh, int lane, int lanes)
{
    if (!sh.staged)
        return;
    const Sim &s = *x.s;
    const int total = sh.total, k = x.sr->k;
    for (int i = lane; i < total; i += lanes)
    {
        // the port and message holding staged frame i (ports without frames are skipped)
        int q = 0;
        while (q + 1 < k && sh.off2[q + 1] <= i)
            q++;
        int link = x.ports[q].in_link;
        const Frame *src = i < sh.off1[q] ? msg_frames(s, x.gt - 2, link) + (i - sh.off2[q])
                                          : msg_frames(s, x.gt - 1, link) + (i - sh.off1[q]);
        frame_load_link(sh.fr()[i], src);
    }
}

// phase 1d (lane q): the window (frames of msg[t-2] from S0 on, of msg[t-1] before E0)
TB_D int sw_phase_window(const SwCtx &x, SwShared &sh, int q)
{
    const int64_t S0 = x.t * SLOT_PS, E0 = S0 + SLOT_PS;
    const int r2 = sh.raw2[q], r1 = sh.raw1[q];
    // index msg[t-2] (window i2 = 0, n2 = r2, n1 = 0), then msg[t-1] (n2 = 0)
    sh.win[q][0] = 0;
    sh.win[q][1] = r2;
    sh.win[q][2] = 0;
    Input all = input_of(x, sh, q);
    int i2 = 0;
    while (i2 < r2 && all.ts(i2) < S0)
        i2++;
    all.n2 = 0;
    int n1 = 0;
    while (n1 < r1 && all.ts(n1) < E0)
        n1++;
    sh.win[q][0] = i2;
    sh.win[q][2] = n1;
    return (r2 - i2) + n1;
}

// the egress port of an arrival (-1: dropped on arrival at a down interface); reads the frame's
// routing fields only
TB_D int sw_egress_for(const SwCtx &x, const Frame &f, int q, int j)
{
    const WorldDesc &wd = *x.wd;
    int ep = wd.n_fail ? epoch_of(wd, f.ts) : 0;
    if (port_down(wd, x.sr->local, q, ep))
        return -1;
    if (x.spray)
        return route_up(wd, x.sr->local, f.dst, x.s->sw_up[x.scratch + (size_t)q * 2 * MAX_TX + j], ep);
    return route(*x.s, wd, x.sr->local, f, ep);
}
TB_D int sw_egress_of(const SwCtx &x, const Input &in, int q, int j)
{
    if (in.smem)
        return sw_egress_for(x, *in.at(j), q, j); // (read in place)
    Frame f;
    frame_load_link(f, in.at(j));
    return sw_egress_for(x, f, q, j);
}
// the region of egress arrivals (times, sources): shared memory when staged
TB_D int64_t *sw_ts_of(const SwCtx &x, SwShared &sh) { return sh.staged ? sh.ets() : x.s->sw_ts + x.scratch; }
TB_D uint32_t *sw_ref_of(const SwCtx &x, SwShared &sh) { return sh.staged ? sh.eref() : x.s->sw_ref + x.scratch; }

// phase 2 (one lane): per-packet ECMP draws, one per forwarded packet in the order the packets
// arrive at the node (all ports merged), from the switch's MRG32k3a stream. (With staged frames
// the warp merges 32-bit keys and computes the draws at once from the stream's look-ahead,
// sw_spray_keyed in tb_kernel.cu, in the same order and with the same values.)
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
            Input in = input_of(x, sh, q);
            if (pos[q] >= in.count())
                continue;
            in.load(f, pos[q]);
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
    Input in = input_of(x, sh, q);
    unsigned dropped = 0;
    int n = in.count();
    for (int j = 0; j < n; j++)
    {
        int e = sw_egress_of(x, in, q, j);
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

// phase 5 (lane e): egress e's region
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
    Input in = input_of(x, sh, q);
    int64_t *ts = sw_ts_of(x, sh);
    uint32_t *ref = sw_ref_of(x, sh);
    int n = in.count();
    for (int j = 0; j < n; j++)
    {
        int e = sw_egress_of(x, in, q, j);
        if (e < 0)
            continue;
        int at = sh.base[e] + sh.rows[q][e]++;
        ts[at] = in.ts(j);
        ref[at] = (uint32_t)(q << 16 | j);
    }
}

// phase 7 (lane e): egress e's arrivals in time order (ties: ns-3's order, insertion sort in
// ingress order), each enqueued (RED) with its arrival event's chain; then the starts of the
// slot. Returns true if the port sent or holds frames.
template <bool PORT_LOCAL>
TB_D bool sw_phase_egress(const SwCtx &x, SwShared &sh, int e, unsigned &ties, unsigned &drops, unsigned &marks,
                          unsigned &ovf)
{
    const Sim &s = *x.s;
    const int n = sh.cnt[e];
    int64_t *ts = sw_ts_of(x, sh) + sh.base[e];
    uint32_t *ref = sw_ref_of(x, sh) + sh.base[e];
    auto load_ref = [&](Frame &f, uint32_t r) { input_of(x, sh, (int)(r >> 16)).load(f, (int)(r & 0xFFFF)); };
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
                bool before;
                if (sh.staged)
                    before = frame_before(*input_of(x, sh, (int)(r >> 16)).at((int)(r & 0xFFFF)),
                                          *input_of(x, sh, (int)(ref[j] >> 16)).at((int)(ref[j] & 0xFFFF)), ties);
                else
                {
                    Frame a, b;
                    load_ref(a, r);
                    load_ref(b, ref[j]);
                    before = frame_before(a, b, ties);
                }
                if (!before)
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
    typename std::conditional<PORT_LOCAL, PortEgress, Egress>::type eg;
    Chain *tx_chain = &pr.last;
    if constexpr (PORT_LOCAL)
    {
        sh.eg_last()[e] = pr.last;
        tx_chain = &sh.eg_last()[e];
    }
    const int out_link = s.H + port;
    eg.open(s.port_ring + (size_t)port * s.ring, s.ring, pr.q_head, pr.q_size, pr.link_free, pr.last_start, tx_chain, pr.red_k, pr.qcap,
            (x.t + 1) * SLOT_PS, s.msg + msg_index(s, x.gt, out_link) * MAX_TX);
    if constexpr (PORT_LOCAL)
        eg.shadow = &sh.eg_tail()[e];
#ifdef TB_QTRACE
    eg.qs = &s;
    eg.qnode = x.wd->H1 + x.sr->local;
    eg.qdev = e + 1;
#endif
    for (int i = 0; i < n; i++)
    {
        Frame p;
        load_ref(p, ref[i]);
        chain_child(p.ch, p.ch, code_arrival(p.len)); // queued: the arrival event's chain
        eg.enqueue(p, p.ts);
    }
    eg.advance(eg.horizon - 1);
    tag_store(&s.msg_tag[msg_index(s, x.gt, out_link)], (int64_t)x.gt << 16 | eg.n_out);
    pr.q_head = eg.head;
    pr.q_size = eg.size;
    pr.link_free = eg.busy_until;
    pr.last_start = eg.began;
    if constexpr (PORT_LOCAL)
        pr.last = *eg.tx_chain;
    drops += eg.drops;
    marks += eg.marks;
    ovf += eg.ovf;
    return eg.n_out > 0 || eg.size > 0;
}

} // namespace tb
