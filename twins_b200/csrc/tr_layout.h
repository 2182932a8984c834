// twins-b200: the RDMA worlds of a run laid out side by side for the slot kernel (plain C++17, on
// the host): hosts of every world, then their switches, ports, links and flows in world order; each
// entity's static record and initial state; the links' rings of arrival buckets; the flows' start
// chains and the order of their roots. The C ABI copies the arrays to the device; the tests' CPU
// harness runs the same slot code over them in host memory.
// (reference: the world packing and device set-up of src/rdma/rmain.cu:1246-1362, 1712-1946)
#pragma once
#include "tb_rng_host.h"
#include "tr_sim.cuh"
#include "tr_world.h"

#include <algorithm>
#include <cmath>
#include <string>
#include <vector>

namespace tr
{

// a run's arrays, with their initial contents (the per-flow and ring arrays that start zeroed are
// only sized: n_flows, n_frames, n_tags, ...)
struct RLayout
{
    int H = 0, S = 0, F = 0, W = 0, P = 0, L = 0;
    int64_t D = 0, max_slots = 0;
    std::vector<RWorld> world;
    std::vector<HostInfo> hinfo;
    std::vector<Nic> nic;
    std::vector<SwInfo> sinfo;
    std::vector<SwState> sw;
    std::vector<PortInfo> pinfo;
    std::vector<Port> port;
    std::vector<uint32_t> rt;
    std::vector<uint8_t> rtp;
    std::vector<FlowInfo> flow;
    std::vector<int> start_list;
    std::vector<uint32_t> root_rank;
    std::vector<LinkInfo> link;
    std::vector<int32_t> txt; // [rate classes][TXT_N]
    std::vector<int> world_hbase, world_fbase;
    size_t n_frames = 0, n_tags = 0;
    int pend_n = 2;
    int ackq_cap = 1024, qps_cap = 1, q0_cap = 64, q3_cap = 4096;
    int max_deg = 1;
    std::string error;
};

constexpr int MAX_FRAMES_PER_BUCKET = 256; // frames a link delivers in one slot, at most

inline RWorld world_params(const RdmaWorldParams &p, int first_flow, int n_flows)
{
    RWorld w{};
    w.nic.mtu = p.mtu;
    w.nic.ack_interval = p.ack_interval;
    w.nic.chunk = p.chunk;
    w.nic.nack_interval = p.nack_interval;
    w.nic.seq_extra = 0;
    w.nic.int_size = p.int_size;
    w.nic.var_win = p.var_win;
    w.nic.ack_high_prio = p.ack_high_prio;
    w.nic.cc = p.cc;
    w.nic.fast_react = p.fast_react;
    w.nic.ns336 = 0;
    w.cc.g = p.g;
    w.cc.rate_first_cnp = p.rate_first_cnp;
    w.cc.clamp = p.clamp;
    w.cc.rpg_threshold = p.rpg_threshold;
    w.cc.rai = p.rai;
    w.cc.rhai = p.rhai;
    w.cc.min_rate = p.min_rate;
    w.cc.dctcp_rai = p.dctcp_rai;
    w.cc.u_target = p.u_target;
    w.cc.mi_thresh = p.mi_thresh;
    w.cc.sample_feedback = p.sample_feedback;
    w.cc.int_multi = p.int_multi;
    w.cc.mtu = p.mtu;
    w.ecn = p.ecn;
    w.qbb = 1;
    w.rate_bound = p.rate_bound;
    w.buffer_size = p.buffer_size;
    w.alpha_int = p.alpha_int;
    w.dec_int = p.dec_int;
    w.rp_int = p.rp_int;
    w.first_flow = first_flow;
    w.n_flows = n_flows;
    return w;
}

// The worlds side by side (each built by build_rdma_world and build_rdma_flows). q3_cap: frames a
// switch port's data queue holds. Returns false (and error) where the run cannot be laid out.
inline bool layout_rdma(RLayout &o, const std::vector<const RdmaWorld *> &worlds, int q3_cap = 4096)
{
    o = RLayout{};
    o.q3_cap = q3_cap;
    const int W = o.W = (int)worlds.size();
    if (W == 0)
        return o.error = "no worlds", false;
    // the slot: the shortest link delay of all worlds
    int64_t D = INT64_MAX;
    for (const RdmaWorld *w : worlds)
        for (int64_t d : w->ldelay)
            D = std::min(D, d);
    if (D <= 0 || D == INT64_MAX)
        return o.error = "a world without links", false;
    o.D = D;
    std::vector<int> hbase(W), sbase(W), lbase(W), fbase(W), pbase_w(W);
    for (int i = 0; i < W; i++)
    {
        const RdmaWorld &w = *worlds[i];
        if (w.P.cc == 1 && (w.P.alpha_int < D || w.P.dec_int < D || w.P.rp_int < D))
            return o.error = "DCQCN timer intervals must be at least the slot (the shortest link delay)", false;
        hbase[i] = o.H, sbase[i] = o.S, lbase[i] = o.L, fbase[i] = o.F, pbase_w[i] = o.P;
        o.H += w.H;
        o.S += w.S;
        o.L += w.L;
        o.F += (int)w.flows.size();
        for (int x = 0; x < w.S; x++)
            o.P += w.deg[w.H + x];
    }
    if (o.H > 65535)
        return o.error = "more than 65535 hosts (frames carry 16-bit host ids)", false;
    o.world_hbase = hbase;
    o.world_fbase = fbase;
    const int H = o.H, S = o.S, F = o.F;
    o.world.resize(W);
    o.hinfo.resize(H);
    o.nic.resize(H);
    o.sinfo.resize(S);
    o.sw.resize(S);
    o.link.resize(o.L);
    o.flow.resize(F);
    o.start_list.assign(F, 0);
    o.root_rank.assign(F, 0);
    std::vector<int> start_off(H + 1, 0);
    std::vector<ChainRun> root_runs_flat;
    std::vector<std::vector<uint32_t>> root_leads(F);
    std::vector<uint32_t> root_of(F);
    std::vector<int> per_nic(H, 0);
    std::vector<uint64_t> rates;
    size_t sl = 0;
    for (int wi = 0; wi < W; wi++)
    {
        const RdmaWorld &w = *worlds[wi];
        o.world[wi] = world_params(w.P, fbase[wi], (int)w.flows.size());
        o.max_slots = std::max(o.max_slots, (int64_t)std::min(w.P.stop_ns / (double)D, 1e15));
        // links: their rings of arrival slots. A frame started in slot k arrives at most
        // 1 + (txmax + delay - 1) / D slots later; a bucket holds what can arrive in a slot at one
        // shortest frame each
        for (int l = 0; l < w.L; l++)
        {
            LinkInfo &x = o.link[lbase[wi] + l];
            x.delay = w.ldelay[l];
            x.bps = w.lbps[l];
            const int64_t txmax = tx_ns(x.bps, w.P.mtu + 128), txmin = tx_ns(x.bps, 60);
            const int64_t nb = 2 + (txmax + x.delay - 1) / D;
            const int64_t cap = txmin == 0 ? MAX_FRAMES_PER_BUCKET : std::min<int64_t>(MAX_FRAMES_PER_BUCKET, D / txmin + 2);
            if (nb > 4096)
                return o.error = "a link's delay is too long for the slot", false;
            x.nb = (uint16_t)nb;
            x.cap = (uint16_t)cap;
            // its rate's row of tx times
            size_t rc = 0;
            while (rc < rates.size() && rates[rc] != x.bps)
                rc++;
            if (rc == rates.size())
            {
                rates.push_back(x.bps);
                for (int b = 0; b < TXT_N; b++)
                    o.txt.push_back((int32_t)tx_ns(x.bps, (uint32_t)b));
            }
            x.rc = (uint32_t)rc;
            x.moff = o.n_frames;
            x.coff = (uint32_t)o.n_tags;
            o.n_frames += (size_t)nb * cap;
            o.n_tags += (size_t)nb;
            o.pend_n = std::max(o.pend_n, (int)nb);
        }
        for (int h = 0; h < w.H; h++)
        {
            HostInfo &hi = o.hinfo[hbase[wi] + h];
            hi.world = wi;
            hi.link_in = lbase[wi] + w.in_link[(size_t)h * w.K];
            hi.link_out = lbase[wi] + w.out_link[(size_t)h * w.K];
            Nic &n = o.nic[hbase[wi] + h];
            n = Nic{};
            n.tc_at = n.ns_at = -1;
            n.ob_last = -(1ll << 16);
            n.due_min = INT64_MAX;
            n.wake = 0;
        }
        const uint32_t rtp_base = (uint32_t)o.rtp.size();
        o.rtp.insert(o.rtp.end(), w.rtp.begin(), w.rtp.end());
        int pb = pbase_w[wi];
        for (int x = 0; x < w.S; x++)
        {
            const int gx = sbase[wi] + x, deg = w.deg[w.H + x];
            SwInfo &si = o.sinfo[gx];
            si.world = wi;
            si.deg = deg;
            si.pbase = pb;
            si.hbase = hbase[wi];
            si.seed = (uint32_t)(w.H + x);
            si.rt_off = (uint32_t)(o.rt.size() / 2);
            o.max_deg = std::max(o.max_deg, deg);
            for (int h = 0; h < w.H; h++)
            {
                o.rt.push_back(w.rt[2 * ((size_t)x * w.H + h)] + rtp_base);
                o.rt.push_back(w.rt[2 * ((size_t)x * w.H + h) + 1]);
            }
            SwState &st = o.sw[gx];
            st = SwState{};
            for (int p = 0; p < deg; p++)
            {
                const RdmaPortCfg &c = w.pcfg[pb - pbase_w[wi] + p];
                PortInfo pi{};
                pi.link_in = lbase[wi] + w.in_link[(size_t)(w.H + x) * w.K + p];
                pi.link_out = lbase[wi] + w.out_link[(size_t)(w.H + x) * w.K + p];
                pi.bps = c.bps;
                pi.hdrm_cap = c.hdrm_cap;
                pi.shift = c.shift;
                pi.kmin = c.kmin;
                pi.kmax = c.kmax;
                pi.pmax = c.pmax;
                o.pinfo.push_back(pi);
                st.mmu.total_hdrm += c.hdrm_cap;
                st.max_shift = c.shift > st.max_shift ? c.shift : st.max_shift;
                Port pt{};
                pt.tc_at = -1;
                pt.ob_last = -(1ll << 16);
                // the port's ECN stream: ConfigEcnStream(port, node * pCnt + device)
                pt.rng = tb::stream_state(1, (uint64_t)(w.H + x) * w.P.ecn_pcnt + (uint64_t)(p + 1), 1);
                o.port.push_back(pt);
            }
            st.mmu.total_rsrv = MMU_RESERVE * (uint32_t)deg;
            pb += deg;
        }
        // flows: ids over all worlds; a root is 1 + the flow's place in its world's start order,
        // offset by the world's first flow
        for (size_t f = 0; f < w.flows.size(); f++)
        {
            const RdmaFlow &x = w.flows[f];
            const int g = fbase[wi] + (int)f;
            FlowInfo &fi = o.flow[g];
            fi = FlowInfo{};
            fi.src = hbase[wi] + x.src;
            fi.dst = hbase[wi] + x.dst;
            fi.size = x.size;
            fi.start = x.start;
            fi.sport = x.sport;
            fi.win = x.win;
            fi.base_rtt = x.base_rtt;
            Chain c{};
            for (size_t i = 0; i < x.runs.size() && i < (size_t)RUNS; i++)
                c.r[i] = ChainRun{x.runs[i].first, x.runs[i].second};
            c.root = (uint32_t)fbase[wi] + x.root;
            c.hash = 0;
            c.tail = 0;
            fi.start_chain = c;
            const int r = (int)c.root - 1;
            root_of[r] = c.root;
            for (size_t i = 0; i < x.runs.size(); i++)
                for (uint32_t k = 0; k < x.runs[i].second; k++)
                    root_leads[r].push_back(x.runs[i].first >> CODE_ORD_BITS);
            per_nic[fi.src]++;
        }
        for (int h = 0; h < w.H; h++)
            start_off[hbase[wi] + h + 1] = w.start_off[h + 1] - w.start_off[h];
        for (size_t f = 0; f < w.start_list.size(); f++)
            o.start_list[sl + f] = fbase[wi] + w.start_list[f];
        sl += w.start_list.size();
    }
    for (int h = 0; h < H; h++)
        start_off[h + 1] += start_off[h];
    for (int h = 0; h < H; h++)
    {
        o.nic[h].next_start = start_off[h];
        o.nic[h].start_end = start_off[h + 1];
    }
    o.qps_cap = std::max(1, *std::max_element(per_nic.begin(), per_nic.end()));
    // the roots in the order of their start chains: the first differing lead (the larger first), a
    // chain that ends first, then the root (reference: src/rdma/rmain.cu:1536-1568)
    std::vector<int> idx(F);
    for (int i = 0; i < F; i++)
        idx[i] = i;
    std::sort(idx.begin(), idx.end(), [&](int a, int b) {
        const std::vector<uint32_t> &x = root_leads[a], &y = root_leads[b];
        for (size_t i = 0; i < x.size() && i < y.size(); i++)
            if (x[i] != y[i])
                return x[i] > y[i];
        if (x.size() != y.size())
            return x.size() < y.size();
        return root_of[a] < root_of[b];
    });
    for (int i = 0; i < F; i++)
        o.root_rank[idx[i]] = (uint32_t)i;
    return true;
}

} // namespace tr
