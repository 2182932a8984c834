// A CPU harness of the RDMA slot code (twins_b200/csrc/tr_sim.cuh), built by tests/test_rdma_sim.py
// with g++: the product's own host and switch slot functions, run an entity at a time over the
// layout of tr_layout.h in host memory, so that their logic can be checked against the oracle's
// fixtures where no GPU is at hand. Test infrastructure: the library runs these functions on the
// GPU (tr_kernel.cu).
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "tr_layout.h"

using namespace tr;

namespace
{
std::string g_err;

template <class T>
T *vec_or_zero(std::vector<T> &v, size_t n)
{
    if (v.size() < n)
        v.resize(n);
    return v.data();
}
} // namespace

extern "C" {

const char *rs_error() { return g_err.c_str(); }

// n worlds (configuration text, topology text, flow file text each); every flow's fct (-1: not
// done) into fct (over all worlds, in world order), the counters into ev[40], the slots run into
// *slots. Returns 0, or -1 with rs_error().
int rs_run(int n, const char **cfg, const char **topo, const char **flows, long long *fct, unsigned long long *ev, long long *slots,
           int tail_log2, int serial_only)
{
    std::vector<RdmaWorld> worlds(n);
    std::vector<const RdmaWorld *> wp;
    for (int i = 0; i < n; i++)
    {
        if (!build_rdma_world(worlds[i], parse_rdma_config(cfg[i]), topo[i], 100000000000ull, 1000) || !build_rdma_flows(worlds[i], flows[i]))
        {
            g_err = worlds[i].error;
            return -1;
        }
        wp.push_back(&worlds[i]);
    }
    RLayout L;
    if (!layout_rdma(L, wp))
    {
        g_err = L.error;
        return -1;
    }
    std::vector<Chain> h_tc(L.H), h_ns(L.H), p_tc(L.P);
    std::vector<Pkt> ackq((size_t)L.H * L.ackq_cap), q0((size_t)L.P * L.q0_cap), q3((size_t)L.P * L.q3_cap);
    std::vector<int> qps((size_t)L.H * L.qps_cap);
    std::vector<Qp> qp(L.F);
    std::vector<QpChains> qc(L.F);
    std::vector<RxQp> rx(L.F);
    std::vector<int64_t> fctv(L.F, -1);
    std::vector<Frame> msg(L.n_frames);
    std::vector<long long> tags(L.n_tags, -(1ll << 16));
    std::vector<unsigned> pend(L.pend_n, 0);
    std::vector<TailNode> tail(1ull << tail_log2);
    unsigned long long tail_cnt = 0;
    std::vector<unsigned long long> evv(EV_N, 0);
    RCtl ctl{};
    RSim s{};
    s.H = L.H, s.S = L.S, s.F = L.F, s.W = L.W, s.P = L.P;
    s.D = L.D;
    s.max_slots = L.max_slots;
    s.world = L.world.data();
    s.hinfo = L.hinfo.data();
    s.nic = L.nic.data();
    s.h_tc = h_tc.data();
    s.h_ns = h_ns.data();
    s.ackq = ackq.data();
    s.ackq_cap = L.ackq_cap;
    s.qps = qps.data();
    s.qps_cap = L.qps_cap;
    s.sinfo = L.sinfo.data();
    s.sw = L.sw.data();
    s.pinfo = L.pinfo.data();
    s.port = L.port.data();
    s.p_tc = p_tc.data();
    s.q0 = q0.data();
    s.q3 = q3.data();
    s.q0_cap = L.q0_cap;
    s.q3_cap = L.q3_cap;
    s.rt = L.rt.data();
    s.rtp = L.rtp.data();
    s.flow = L.flow.data();
    s.start_list = L.start_list.data();
    s.root_rank = L.root_rank.data();
    s.qp = qp.data();
    s.qc = qc.data();
    s.rx = rx.data();
    s.fct = fctv.data();
    s.link = L.link.data();
    s.txt = L.txt.data();
    s.msg = msg.data();
    s.msg_cnt = tags.data();
    s.pend = pend.data();
    s.pend_n = L.pend_n;
    s.tail = tail.data();
    s.tail_cnt = &tail_cnt;
    s.tail_mask = (1ull << tail_log2) - 1;
    s.ev = evv.data();
    s.ctl = &ctl;
    s.serial_only = serial_only;
    std::vector<SwPort> ports(L.max_deg);
    std::vector<SArr> arr(SW_STAGE > HOST_STAGE ? SW_STAGE : HOST_STAGE);
    std::vector<uint16_t> ord(SW_STAGE);
    std::vector<Frame> fr(SW_FRAMES);
    std::vector<HPre> hpre(HOST_STAGE);
    int flags[4];
    const SwWork work{ports.data(), fr.data(), arr.data(), ord.data(), flags};
    Due due[MAX_DUE];
    while (!ctl.finished)
    {
        const int64_t t = ctl.slot;
        unsigned act = 0;
        unsigned long long wake = ~0ull;
        for (int h = 0; h < L.H; h++)
        {
            int64_t w = INT64_MAX;
            if (host_slot(s, h, t, &w, due, arr.data(), hpre.data(), 0, 1))
                act++;
            if (w != INT64_MAX && (unsigned long long)w < wake)
                wake = (unsigned long long)w;
        }
        for (int x = 0; x < L.S; x++)
            if (switch_slot(s, x, t, work, 0, 1))
                act++;
        slot_close(s, t, act, wake, ctl.flows_done);
    }
    for (int f = 0; f < L.F; f++)
        fct[f] = fctv[f];
    memcpy(ev, evv.data(), sizeof(unsigned long long) * EV_N);
    *slots = ctl.slot;
    return 0;
}

} // extern "C"
