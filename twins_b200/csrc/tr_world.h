// twins-b200: an RDMA world's set-up on the host (plain C++17): the HPCC fork's parameters from its
// KEY VALUE configuration, the topology (TwiNS's "hosts / switches / link" format), the link
// wiring and port numbering, the switches' ECMP route tables (ns-3's CalculateRoute: BFS from each
// host), maxRtt / maxBdp (the window and base RTT of every flow under GLOBAL_T), and each switch
// port's PFC headroom and threshold shift and ECN thresholds; and the flows with their source ports,
// start order and start chains. Equal, field by field, to the reference's build_world
// (src/rdma/rmain.cu:364-1021), which the oracle's digests pin.
#pragma once
#include <algorithm>
#include <climits>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <map>
#include <sstream>
#include <string>
#include <vector>

namespace tr
{

using RdmaConfig = std::map<std::string, std::vector<std::string>>;

// an event's code in a chain: (lead + 1) << 5 | (31 - ordinal), both saturating (as
// tr_chain.cuh's event_code, which device code uses)
inline uint32_t start_code(int64_t lead, int ord)
{
    uint64_t l = (uint64_t)lead + 1;
    const uint64_t most = (1ull << 27) - 2;
    if (l > most)
        l = most;
    return (uint32_t)(l << 5 | (31u - (uint32_t)(ord < 31 ? ord : 31)));
}

// "KEY v1 v2 ..." per line (reference: src/rdma/rmain.cu:111-135)
inline RdmaConfig parse_rdma_config(const std::string &text)
{
    RdmaConfig cfg;
    std::istringstream lines(text);
    std::string line;
    while (std::getline(lines, line))
    {
        std::istringstream is(line);
        std::string key, v;
        if (!(is >> key))
            continue;
        std::vector<std::string> vals;
        while (is >> v)
            vals.push_back(v);
        cfg[key] = vals;
    }
    return cfg;
}

// "50Mb/s", "100Gbps": the number times 10^3 (K, k), 10^6 (M) or 10^9 (G), truncated (reference:
// src/rdma/rmain.cu:146-161)
inline uint64_t parse_rate(const std::string &s)
{
    size_t i = 0;
    while (i < s.size() && (isdigit((unsigned char)s[i]) || s[i] == '.'))
        i++;
    const double v = atof(s.substr(0, i).c_str());
    const char u = i < s.size() ? s[i] : 0;
    const double m = u == 'K' || u == 'k' ? 1e3 : u == 'M' ? 1e6 : u == 'G' ? 1e9 : 1;
    return (uint64_t)(v * m);
}

struct RdmaWorldParams
{
    int cc, int_size;
    uint32_t mtu, ack_interval, chunk;
    int64_t nack_interval;
    uint64_t bps;
    int64_t delay;
    double stop_ns; // SIMULATOR_STOP_TIME in ns: the run stops at slot stop_ns / slot length
    uint32_t win;
    uint64_t base_rtt;
    int var_win, rate_bound, ack_high_prio, ecn;
    int64_t alpha_int, dec_int, rp_int;
    uint32_t rpg_threshold;
    uint64_t rai, rhai, min_rate, dctcp_rai;
    uint32_t mi_thresh;
    int fast_react, sample_feedback;
    uint32_t int_multi, buffer_size, ecn_pcnt;
    double g, rate_first_cnp, u_target;
    int clamp; // CLAMP_TARGET_RATE
};

struct RdmaPortCfg
{
    uint64_t bps;
    uint32_t hdrm_cap, shift, kmin, kmax;
    double pmax;
};

// a flow as the set-up leaves it: its ends, size and start, source port (per host pair from 10000,
// in start order), place in start order, window and base RTT, devices, and the chain of its
// StartApplication (root = 1 + its place; runs newest first, as tr_chain.cuh reads them)
struct RdmaFlow
{
    int src, dst;
    uint64_t size;
    int64_t start;
    uint32_t sport, order, win;
    uint64_t base_rtt;
    uint32_t snic, rnic, root;
    std::vector<std::pair<uint32_t, uint32_t>> runs;
};

struct RdmaWorld
{
    RdmaWorldParams P{};
    int H = 0, S = 0, N = 0, L = 0, K = 1;
    std::vector<int> deg, out_link, in_link, link_dst, link_dport; // [N K]; links' far ends [L]
    std::vector<uint64_t> lbps;                                     // [L]
    std::vector<int64_t> ldelay;                                    // [L]
    std::vector<uint32_t> rt;                                       // [S H] (first port, count)
    std::vector<uint8_t> rtp;                                       // the route tables' ports
    std::vector<RdmaPortCfg> pcfg;                                  // every switch's ports in turn
    std::vector<RdmaFlow> flows;                                    // in file order
    std::vector<int> start_list, start_off;                         // per host, its flows in start order
    std::string error;
};

// The flows of a flow file ("src,dst,flow_size,start_ns" after a header line; lines that do not
// parse are skipped) in a world made by build_rdma_world (reference: src/rdma/rmain.cu:842-1021,
// for hosts of one link). ns-3 starts them through one ScheduleFlowInputs event per start time,
// each scheduled by the previous one (or by main), then Application::Start, then StartApplication:
// their start chains.
inline bool finish_rdma_flows(RdmaWorld &w);

inline bool build_rdma_flows(RdmaWorld &w, const std::string &csv)
{
    std::istringstream f(csv);
    std::string line;
    std::getline(f, line);
    w.flows.clear();
    while (std::getline(f, line))
    {
        long long a, b;
        unsigned long long sz, st;
        if (sscanf(line.c_str(), "%lld,%lld,%llu,%llu", &a, &b, &sz, &st) != 4)
            continue;
        if (a < 0 || b < 0 || a > INT_MAX || b > INT_MAX)
            return w.error = "a flow with a negative or out-of-range node id", false;
        RdmaFlow x{};
        x.src = (int)a, x.dst = (int)b, x.size = sz, x.start = (int64_t)st;
        w.flows.push_back(x);
    }
    return finish_rdma_flows(w);
}

// the same from arrays (a flow file's columns)
inline bool build_rdma_flows(RdmaWorld &w, int n, const int *src, const int *dst, const long long *size, const long long *start_ns)
{
    w.flows.clear();
    for (int i = 0; i < n; i++)
    {
        if (src[i] < 0 || dst[i] < 0 || size[i] < 0 || start_ns[i] < 0)
            return w.error = "a flow with a negative node id, size or start", false;
        RdmaFlow x{};
        x.src = src[i], x.dst = dst[i], x.size = (uint64_t)size[i], x.start = start_ns[i];
        w.flows.push_back(x);
    }
    return finish_rdma_flows(w);
}

// the flows read: their checks, source ports, start order and chains, the hosts' start lists
inline bool finish_rdma_flows(RdmaWorld &w)
{
    const int F = (int)w.flows.size(), H = w.H;
    for (RdmaFlow &x : w.flows)
    {
        if (x.src >= H || x.dst >= H)
            return w.error = "a flow between nodes that are not hosts", false;
        x.win = w.P.win;
        x.base_rtt = w.P.base_rtt;
    }
    std::vector<int> order(F);
    for (int i = 0; i < F; i++)
        order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return w.flows[a].start < w.flows[b].start; });
    std::map<std::pair<int, int>, uint32_t> port;
    int64_t prev_t = 0;
    int prev_n = 0, k = 0;
    for (int i = 0; i < F;)
    {
        int j = i;
        while (j < F && w.flows[order[j]].start == w.flows[order[i]].start)
            j++;
        const int64_t t = w.flows[order[i]].start;
        for (int m = i; m < j; m++)
        {
            RdmaFlow &x = w.flows[order[m]];
            auto it = port.emplace(std::make_pair(x.src, x.dst), 10000u).first;
            x.sport = it->second++;
            x.order = (uint32_t)m;
            x.root = (uint32_t)(m + 1);
            // its start chain: three events, newest first, equal codes in one run
            const uint32_t codes[3] = {start_code(t - prev_t, k == 0 ? 0 : prev_n), start_code(0, m - i), start_code(0, 0)};
            x.runs.clear();
            for (uint32_t c : codes)
                if (!x.runs.empty() && x.runs.front().first == c)
                    x.runs.front().second++;
                else
                    x.runs.insert(x.runs.begin(), {c, 1u});
        }
        prev_t = t;
        prev_n = j - i;
        k++;
        i = j;
    }
    w.start_list.assign(F, 0);
    w.start_off.assign(H + 1, 0);
    for (int i = 0; i < F; i++)
        w.start_off[w.flows[order[i]].src + 1]++;
    for (int h = 0; h < H; h++)
        w.start_off[h + 1] += w.start_off[h];
    std::vector<int> pos(w.start_off.begin(), w.start_off.end() - 1);
    for (int i = 0; i < F; i++)
        w.start_list[pos[w.flows[order[i]].src]++] = order[i];
    return true;
}

// The world of a configuration and a topology, every link at bps with delay ns. Returns false
// (and error) where the reference refuses it.
inline bool build_rdma_world(RdmaWorld &w, const RdmaConfig &cfg, const std::string &topo, uint64_t bps, int64_t delay)
{
    auto has = [&](const char *k) { return cfg.count(k) && !cfg.at(k).empty(); };
    auto str = [&](const char *k, const std::string &d) { return has(k) ? cfg.at(k)[0] : d; };
    auto num = [&](const char *k, double d) { return has(k) ? atof(cfg.at(k)[0].c_str()) : d; };
    auto u32 = [&](const char *k, uint32_t d) { return has(k) ? (uint32_t)strtoul(cfg.at(k)[0].c_str(), 0, 10) : d; };
    RdmaWorldParams &P = w.P;
    P = RdmaWorldParams{};
    P.cc = (int)u32("CC_MODE", 1);
    if (P.cc != 1 && P.cc != 3 && P.cc != 8)
        return w.error = "CC_MODE: only 1 (DCQCN), 3 (HPCC) and 8 (DCTCP)", false;
    if (u32("MULTI_RATE", 1) && P.cc == 3)
        return w.error = "MULTI_RATE 1", false;
    if (u32("L2_BACK_TO_ZERO", 0))
        return w.error = "L2_BACK_TO_ZERO 1", false;
    P.int_size = P.cc == 3 ? 42 : 0;
    P.mtu = u32("PACKET_PAYLOAD_SIZE", 1000);
    P.ack_interval = u32("L2_ACK_INTERVAL", 0);
    P.chunk = u32("L2_CHUNK_SIZE", 0);
    if (P.ack_interval == 0)
        return w.error = "L2_ACK_INTERVAL 0", false;
    P.nack_interval = 500000; // (the NACK generation interval, 500 us)
    P.delay = delay;
    P.var_win = (int)u32("VAR_WIN", 0);
    P.rate_bound = (int)u32("RATE_BOUND", 1);
    P.ack_high_prio = (int)u32("ACK_HIGH_PRIO", 0);
    P.ecn = (int)u32("ENABLE_QCN", 1);
    P.g = num("EWMA_GAIN", 1.0 / 16);
    P.rate_first_cnp = 1.0;
    P.clamp = (int)u32("CLAMP_TARGET_RATE", 0);
    // (MicroSeconds of an integer: the attributes are doubles)
    P.alpha_int = (int64_t)(uint64_t)num("ALPHA_RESUME_INTERVAL", 55) * 1000;
    P.dec_int = (int64_t)(uint64_t)num("RATE_DECREASE_INTERVAL", 4) * 1000;
    P.rp_int = (int64_t)(uint64_t)num("RP_TIMER", 1500) * 1000;
    P.rpg_threshold = u32("FAST_RECOVERY_TIMES", 5);
    P.rai = parse_rate(str("RATE_AI", "5Mb/s"));
    P.rhai = parse_rate(str("RATE_HAI", "50Mb/s"));
    P.min_rate = parse_rate(str("MIN_RATE", "100Mb/s"));
    P.dctcp_rai = parse_rate(str("DCTCP_RATE_AI", "1000Mb/s"));
    P.u_target = num("U_TARGET", 0.95);
    P.mi_thresh = u32("MI_THRESH", 5);
    P.fast_react = (int)u32("FAST_REACT", 1);
    P.sample_feedback = (int)u32("SAMPLE_FEEDBACK", 0);
    P.int_multi = u32("INT_MULTI", 1);
    P.buffer_size = u32("BUFFER_SIZE", 16) * 1024 * 1024;
    P.ecn_pcnt = 257;
    if (u32("GLOBAL_T", 1) != 1)
        return w.error = "GLOBAL_T 0 (SimAI topologies only)", false;
    // (in double, as the reference converts it: reference src/rdma/rmain.cu:526)
    P.stop_ns = num("SIMULATOR_STOP_TIME", 10.0) * 1e9;

    // ---- topology: hosts h0.., switches s0..; nodes are hosts, then switches
    std::vector<std::pair<int, int>> links;
    {
        std::istringstream f(topo);
        std::string x, a, b;
        while (f >> x)
            if (x == "hosts")
                f >> w.H;
            else if (x == "switches")
                f >> w.S;
            else if (x == "link")
            {
                if (!(f >> a >> b))
                    return w.error = "a link line without two ends", false;
                // h<i> (0 <= i < hosts) or s<j> (0 <= j < switches), after the hosts and switches lines
                auto id = [&](const std::string &y) -> int {
                    if (y.size() < 2 || (y[0] != 'h' && y[0] != 's'))
                        return -1;
                    char *end = nullptr;
                    const long v = strtol(y.c_str() + 1, &end, 10);
                    if (*end || v < 0 || v >= (y[0] == 'h' ? w.H : w.S))
                        return -1;
                    return (y[0] == 'h' ? 0 : w.H) + (int)v;
                };
                const int ia = id(a), ib = id(b);
                if (ia < 0 || ib < 0)
                    return w.error = "a link to a node that does not exist (or before its hosts / switches line)", false;
                links.push_back({ia, ib});
            }
    }
    if (w.H <= 0 || w.S < 0)
        return w.error = "no hosts", false;
    const int H = w.H, S = w.S, N = w.N = H + S, L = w.L = 2 * (int)links.size();
    P.bps = bps;
    w.deg.assign(N, 0);
    for (auto &l : links)
        w.deg[l.first]++, w.deg[l.second]++;
    int K = 1;
    for (int n = 0; n < N; n++)
        K = std::max(K, w.deg[n]);
    w.K = K;
    if (K > 256)
        return w.error = "a node has more than 256 ports", false;
    for (int h = 0; h < H; h++)
        if (w.deg[h] != 1)
            return w.error = "a host without exactly one link", false;
    w.out_link.assign((size_t)N * K, -1);
    w.in_link.assign((size_t)N * K, -1);
    w.link_dst.assign(L, 0);
    w.link_dport.assign(L, 0);
    w.lbps.assign(L, bps);
    w.ldelay.assign(L, delay);
    // ports in link order; link i is 2i from its first node to its second, 2i + 1 back; a node's
    // neighbours by id (with two links to one neighbour, the last one's port)
    std::vector<std::map<int, int>> nbr(N);
    {
        std::vector<int> d(N, 0);
        for (size_t i = 0; i < links.size(); i++)
        {
            const int a = links[i].first, b = links[i].second, pa = d[a]++, pb = d[b]++;
            w.out_link[(size_t)a * K + pa] = (int)(2 * i);
            w.in_link[(size_t)a * K + pa] = (int)(2 * i + 1);
            w.out_link[(size_t)b * K + pb] = (int)(2 * i + 1);
            w.in_link[(size_t)b * K + pb] = (int)(2 * i);
            w.link_dst[2 * i] = b, w.link_dport[2 * i] = pb;
            w.link_dst[2 * i + 1] = a, w.link_dport[2 * i + 1] = pa;
            nbr[a][b] = pa;
            nbr[b][a] = pb;
        }
    }
    // ---- routes: a BFS from every host over the switches; a switch's next hops towards the host are
    // the nodes one hop nearer, in the order the BFS reaches them (neighbours by id); path delay,
    // per-hop tx time of one MTU frame and the slowest link, summed along the path that first
    // reaches a host
    std::vector<std::vector<int>> next(S);
    std::vector<std::vector<uint8_t>> ports((size_t)S * H);
    uint64_t max_rtt = 0, max_bdp = 0;
    int far = 0; // the most links on a path between hosts
    for (int h = 0; h < H; h++)
    {
        std::vector<int> q = {h}, dis(N, -1);
        std::vector<uint64_t> dl(N, 0), txd(N, 0), bw(N, 0);
        dis[h] = 0;
        bw[h] = ~0ull;
        for (size_t i = 0; i < q.size(); i++)
        {
            const int now = q[i], d = dis[now];
            for (auto &e : nbr[now])
            {
                const int nx = e.first;
                if (dis[nx] < 0)
                {
                    const int l = w.out_link[(size_t)now * K + e.second];
                    dis[nx] = d + 1;
                    dl[nx] = dl[now] + (uint64_t)w.ldelay[l];
                    txd[nx] = txd[now] + (uint64_t)P.mtu * 1000000000ull * 8 / w.lbps[l];
                    bw[nx] = std::min(bw[now], w.lbps[l]);
                    if (nx >= H)
                        q.push_back(nx);
                }
                if (d + 1 == dis[nx] && nx >= H)
                    next[nx - H].push_back(now);
            }
        }
        for (int i = 0; i < H; i++)
        {
            far = std::max(far, dis[i]);
            // maxRtt: delay * 2 + txDelay; maxBdp: its product with the slowest link's rate
            const uint64_t rtt = dl[i] * 2 + txd[i];
            max_rtt = std::max<uint64_t>(max_rtt, rtt);
            max_bdp = std::max<uint64_t>(max_bdp, rtt * bw[i] / 1000000000ull / 8);
        }
        for (int x = 0; x < S; x++)
        {
            for (int y : next[x])
                ports[(size_t)x * H + h].push_back((uint8_t)nbr[H + x][y]);
            next[x].clear();
        }
    }
    if (P.cc == 3 && far - 1 > 5)
        return w.error = "HPCC: a path of more than 5 switches (INT records 5)", false;
    w.rt.assign((size_t)S * H * 2, 0);
    for (int x = 0; x < S; x++)
        for (int h = 0; h < H; h++)
        {
            const auto &v = ports[(size_t)x * H + h];
            w.rt[2 * ((size_t)x * H + h)] = (uint32_t)w.rtp.size();
            w.rt[2 * ((size_t)x * H + h) + 1] = (uint32_t)v.size();
            w.rtp.insert(w.rtp.end(), v.begin(), v.end());
        }
    P.base_rtt = max_rtt;
    const uint32_t has_win = u32("HAS_WIN", 1);
    P.win = has_win ? (uint32_t)max_bdp : 0;
    // a server's world with the whole cluster's maxRtt and maxBdp (reference: src/rdma/rmain.cu:687-690)
    if (u32("NVL_BASE_RTT", 0))
        P.base_rtt = u32("NVL_BASE_RTT", 0);
    if (u32("NVL_WIN", 0) && has_win)
        P.win = u32("NVL_WIN", 0);
    // ---- switch ports: headroom 3 x rate x delay; the PFC threshold's shift from 3, one less per
    // halving of the rate above the NIC's (host 0's link); ECN thresholds (KB) and probability by rate
    const uint64_t nic_rate = w.lbps[w.out_link[0]];
    auto ecn = [&](const char *key, uint64_t rate, double *out) {
        if (!has(key))
            return false;
        const std::vector<std::string> &v = cfg.at(key);
        const int n = atoi(v[0].c_str());
        for (int i = 0; i < n; i++)
            if (strtoull(v[1 + 2 * i].c_str(), 0, 10) == rate)
            {
                *out = atof(v[2 + 2 * i].c_str());
                return true;
            }
        return false;
    };
    for (int x = 0; x < S; x++)
        for (int p = 0; p < w.deg[H + x]; p++)
        {
            const int l = w.out_link[(size_t)(H + x) * K + p];
            RdmaPortCfg pc{};
            uint64_t r = w.lbps[l];
            pc.bps = r;
            pc.hdrm_cap = (uint32_t)(r * (uint64_t)w.ldelay[l] / 8 / 1000000000ull * 3);
            pc.shift = 3;
            while (r > nic_rate && pc.shift > 0)
            {
                pc.shift--;
                r /= 2;
            }
            double kmin = 0, kmax = 0, pmax = 0;
            if (!ecn("KMIN_MAP", pc.bps, &kmin) || !ecn("KMAX_MAP", pc.bps, &kmax) || !ecn("PMAX_MAP", pc.bps, &pmax))
                return w.error = "KMIN/KMAX/PMAX_MAP: no entry for a port's rate", false;
            pc.kmin = (uint32_t)kmin * 1000;
            pc.kmax = (uint32_t)kmax * 1000;
            pc.pmax = pmax;
            w.pcfg.push_back(pc);
        }
    return true;
}

} // namespace tr
