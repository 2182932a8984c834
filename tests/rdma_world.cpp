// A C shim over the RDMA world set-up (twins_b200/csrc/tr_world.h), built by
// tests/test_rdma_world.py with g++: the world as JSON, in the fields and order of the oracle's
// oracle/rdma_world_kat.cpp.
#include <cstdio>
#include <cstdarg>
#include <cstring>

#include "tr_world.h"

using namespace tr;

namespace
{
std::string out;

void add(const char *fmt, ...) __attribute__((format(printf, 1, 2)));
void add(const char *fmt, ...)
{
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    out += buf;
}

template <typename T>
void arr(const char *key, const std::vector<T> &v, bool comma = true)
{
    add("\"%s\":[", key);
    for (size_t i = 0; i < v.size(); i++)
        add("%s%lld", i ? "," : "", (long long)v[i]);
    add("]%s", comma ? "," : "");
}
} // namespace

extern "C" {

// the world of a configuration, a topology (100 Gb/s, 1 us links) and a flow file as JSON; NULL
// and the reason in *err where it is refused
const char *rw_world(const char *config, const char *topo, const char *flows, const char **err)
{
    RdmaWorld w;
    out.clear();
    if (!build_rdma_world(w, parse_rdma_config(config), topo, 100000000000ull, 1000) || !build_rdma_flows(w, flows))
    {
        out = w.error;
        *err = out.c_str();
        return nullptr;
    }
    const RdmaWorldParams &P = w.P;
    add("{\"params\":[%d,%d,%u,%u,%u,%lld,%llu,%lld,%u,%llu,%d,%d,%d,%d,%lld,%lld,%lld,%u,%llu,%llu,%llu,%llu,%u,%d,%d,%u,%u,%u],", P.cc,
        P.int_size, P.mtu, P.ack_interval, P.chunk, (long long)P.nack_interval, (unsigned long long)P.bps, (long long)P.delay, P.win,
        (unsigned long long)P.base_rtt, P.var_win, P.rate_bound, P.ack_high_prio, P.ecn, (long long)P.alpha_int, (long long)P.dec_int,
        (long long)P.rp_int, P.rpg_threshold, (unsigned long long)P.rai, (unsigned long long)P.rhai, (unsigned long long)P.min_rate,
        (unsigned long long)P.dctcp_rai, P.mi_thresh, P.fast_react, P.sample_feedback, P.int_multi, P.buffer_size, P.ecn_pcnt);
    add("\"params_f\":[\"%a\",\"%a\",\"%a\"],", P.g, P.rate_first_cnp, P.u_target);
    add("\"dims\":[%d,%d,%d,%d,%d],", w.H, w.S, w.N, w.L, w.K);
    arr("deg", w.deg);
    arr("out_link", w.out_link);
    arr("in_link", w.in_link);
    arr("link_dst", w.link_dst);
    arr("link_dport", w.link_dport);
    arr("lbps", w.lbps);
    arr("ldelay", w.ldelay);
    arr("rt", w.rt);
    arr("rtp", w.rtp);
    std::vector<long long> pc;
    add("\"pcfg_pmax\":[");
    for (size_t i = 0; i < w.pcfg.size(); i++)
    {
        const RdmaPortCfg &c = w.pcfg[i];
        pc.push_back((long long)c.bps), pc.push_back(c.hdrm_cap), pc.push_back(c.shift), pc.push_back(c.kmin), pc.push_back(c.kmax);
        add("%s\"%a\"", i ? "," : "", c.pmax);
    }
    add("],");
    arr("pcfg", pc);
    add("\"flows\":[");
    for (size_t i = 0; i < w.flows.size(); i++)
    {
        const RdmaFlow &x = w.flows[i];
        add("%s[%d,%d,%llu,%lld,%u,%u,%u,%llu,%u,%u,%u", i ? "," : "", x.src, x.dst, (unsigned long long)x.size, (long long)x.start, x.sport,
            x.order, x.win, (unsigned long long)x.base_rtt, x.snic, x.rnic, x.root);
        for (auto &r : x.runs)
            add(",%u,%u", r.first, r.second);
        add("]");
    }
    add("],");
    arr("start_list", w.start_list);
    arr("start_off", w.start_off, false);
    add("}");
    *err = nullptr;
    return out.c_str();
}
}
