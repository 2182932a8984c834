// Test infrastructure, not product code: the reference's RDMA world set-up, printed.
//
// Built by `make -C oracle ref-rdma-world` from the reference's own src/rdma/rmain.cu (its main
// renamed away; the CPU build of rdma_cpu/rdma/island.h): for a config, a topology file and a flow
// file, it runs the reference's build_world and prints, as one JSON object, the world's parameters,
// its link wiring, its switches' ECMP route tables and port configurations, maxRtt / maxBdp, and
// its flows (in file order, with their ports, start order and start chains) and start lists.
// tests/golden/make_rdma_fixtures.py stores a digest of each field per world, against which
// tests/test_rdma_world.py checks twins_b200/csrc/tr_world.h.
#define main twins_rdma_main
#include "rdma/rmain.cu"
#undef main

template <typename T>
static void arr(const char *key, const std::vector<T> &v, bool comma = true)
{
    printf("\"%s\":[", key);
    for (size_t i = 0; i < v.size(); i++)
        printf("%s%lld", i ? "," : "", (long long)v[i]);
    printf("]%s", comma ? "," : "");
}

int main(int argc, char **argv)
{
    if (argc < 4)
    {
        fprintf(stderr, "usage: rdma_world_kat CONFIG TOPO FLOWS\n");
        return 2;
    }
    Config cfg;
    if (!read_config(argv[1], cfg))
        return 1;
    World w;
    w.name = "kat";
    if (!build_world(w, cfg, argv[2], argv[3], 100000000000ull, 1000))
        return 1;
    const Params &P = w.P;
    printf("{\"params\":[%d,%d,%u,%u,%u,%lld,%llu,%lld,%u,%llu,%d,%d,%d,%d,%lld,%lld,%lld,%u,%llu,%llu,%llu,%llu,%u,%d,%d,%u,%u,%u],", P.cc,
           P.int_size, P.mtu, P.ack_interval, P.chunk, (long long)P.nack_interval, (unsigned long long)P.bps, (long long)P.delay, P.win,
           (unsigned long long)P.base_rtt, P.var_win, P.rate_bound, P.ack_high_prio, P.ecn, (long long)P.alpha_int, (long long)P.dec_int,
           (long long)P.rp_int, P.rpg_threshold, (unsigned long long)P.rai, (unsigned long long)P.rhai, (unsigned long long)P.min_rate,
           (unsigned long long)P.dctcp_rai, P.mi_thresh, P.fast_react, P.sample_feedback, P.int_multi, P.buffer_size, P.ecn_pcnt);
    printf("\"params_f\":[\"%a\",\"%a\",\"%a\"],", P.g, P.rate_first_cnp, P.u_target);
    printf("\"dims\":[%d,%d,%d,%d,%d],", w.H, w.S, w.N, w.L, w.K);
    arr("deg", w.deg);
    arr("out_link", w.out_link);
    arr("in_link", w.in_link);
    arr("link_dst", w.link_dst);
    arr("link_dport", w.link_dport);
    arr("lbps", w.lbps);
    arr("ldelay", w.ldelay);
    std::vector<long long> rt;
    for (const Route &r : w.rt)
        rt.push_back(r.off), rt.push_back(r.n);
    arr("rt", rt);
    arr("rtp", w.rtp);
    std::vector<long long> pc;
    printf("\"pcfg_pmax\":[");
    for (size_t i = 0; i < w.pcfg.size(); i++)
    {
        const PortCfg &c = w.pcfg[i];
        pc.push_back((long long)c.bps), pc.push_back(c.hdrm_cap), pc.push_back(c.shift), pc.push_back(c.kmin), pc.push_back(c.kmax);
        printf("%s\"%a\"", i ? "," : "", c.pmax);
    }
    printf("],");
    arr("pcfg", pc);
    // flows: src, dst, size, start, sport, order, win, base_rtt, snic, rnic, then their start
    // chains' root and runs (code, count), newest first
    printf("\"flows\":[");
    for (size_t i = 0; i < w.fi.size(); i++)
    {
        const FlowInfo &x = w.fi[i];
        printf("%s[%d,%d,%llu,%lld,%u,%u,%u,%llu,%u,%u,%u", i ? "," : "", x.src, x.dst, (unsigned long long)x.size, (long long)x.start, x.sport,
               x.order, x.win, (unsigned long long)x.base_rtt, x.snic, x.rnic, x.start_chain.root);
        for (int r = 0; r < RUNS && x.start_chain.r[r].code; r++)
            printf(",%u,%u", x.start_chain.r[r].code, x.start_chain.r[r].cnt);
        printf("]");
    }
    printf("],");
    arr("start_list", w.start_list);
    arr("start_off", w.start_off, false);
    printf("}\n");
    return 0;
}
