// twins: the reference's command line (src/main.cu:139-264) over the twins-b200 C ABI.
//   twins (--k=<4..32> | --topo=leafspine --leaves=L --spines=S --hpl=N | --topo=graph --topofile=F
//          [--fail=T:sA:sB[:up],...]) (--flows=<csv> [--out=csv] | --worlds=<file>)
//         [--tcp=dctcp|newreno|cubic] [--ecnK=30] [--queue=200] [--fin=0|1] [--spray=0|1]
//         [--RngSeed=1] [--RngRun=1] [--ecmp_from=csv [--hash_check=1]] [--max_slots=N]
//         [--host_lanes=N] [--hbm_budget_gb=G] [--qtrace=F --qtrace_until=ps [--qtrace_from=ps]]
// --qtrace: every enqueue with from <= time < until (ps), as the reference writes it
// (src/main.cu:1077-1100); recorded by the trace build, which this front-end runs (twins-trace)
// when it was built without it.
// A worlds file holds one world per line: flows=..,tcp=..,ecnK=..,queue=..,fin=..,ecmp_from=..,out=..
// Output: fct.csv per world (src,dst,flow_size,start_ns,established_ns,completed_ns); stdout:
// "Simulation Duration", "Executed Slots" and a counter line, as the reference prints them.
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <unistd.h>
#include <vector>

#include "../../include/twinsb200.h"

namespace
{

struct Flows
{
    std::vector<int> src, dst;
    std::vector<long long> size, start, conn;
};

bool load_flows(const std::string &path, int H, Flows &f)
{
    std::ifstream in(path);
    if (!in)
        return false;
    std::string line;
    while (std::getline(in, line))
    {
        if (line.empty() || !isdigit((unsigned char)line[0]))
            continue;
        std::stringstream ss(line);
        std::vector<long long> v;
        for (std::string x; std::getline(ss, x, ',');)
            v.push_back(std::stoll(x));
        if (v.size() < 3)
            continue;
        f.src.push_back((int)v[0]);
        if (v.size() == 3)
        {
            f.dst.push_back((int)((v[0] + H / 2) % H)); // GeDES pairing: host i with i + H/2
            f.size.push_back(v[1]);
            f.start.push_back(v[2]);
            f.conn.push_back(-1);
        }
        else
        {
            f.dst.push_back((int)v[1]);
            f.size.push_back(v[2]);
            f.start.push_back(v[3]);
            f.conn.push_back(v.size() >= 5 ? v[4] : -1);
        }
    }
    return true;
}

bool load_hashes(const std::string &path, size_t n, std::vector<unsigned> &hd, std::vector<unsigned> &ha)
{
    std::ifstream in(path);
    if (!in)
        return false;
    std::string line;
    std::getline(in, line);
    while (hd.size() < n && std::getline(in, line))
    {
        std::vector<std::string> v;
        std::stringstream ss(line);
        for (std::string x; std::getline(ss, x, ',');)
            v.push_back(x);
        if (v.size() < 8)
            return false;
        hd.push_back((unsigned)std::stoul(v[6]));
        ha.push_back((unsigned)std::stoul(v[7]));
    }
    return hd.size() == n;
}

int tcp_of(const std::string &t) { return t == "dctcp" ? TB_TCP_DCTCP : t == "newreno" ? TB_TCP_NEWRENO : t == "cubic" ? TB_TCP_CUBIC : -1; }

struct World
{
    std::string flows, ecmp_from, out;
    int tcp, ecn_k, queue, fin;
};

} // namespace

int main(int argc, char **argv)
{
    int k = 4, leaves = 16, spines = 8, hpl = 16, ecn_k = 30, queue = 200, fin = 0, spray = 0, hash_check = 0, host_lanes = 0;
    long long seed = 1, run = 1, max_slots = 2000000, qtrace_from = 0, qtrace_until = 0;
    std::string qtrace_file;
    double budget_gb = 0;
    std::string flow_file, out = "fct.csv", tcp = "dctcp", topo = "fattree", topofile, fail_spec, worlds_file, ecmp_from;
    for (int i = 1; i < argc; i++)
    {
        std::string a = argv[i];
        auto has = [&](const char *p) { return a.rfind(p, 0) == 0; };
        auto val = [&](const char *p) { return a.substr(strlen(p)); };
        if (has("--k="))
            k = std::stoi(val("--k="));
        else if (has("--flows="))
            flow_file = val("--flows=");
        else if (has("--out="))
            out = val("--out=");
        else if (has("--tcp="))
            tcp = val("--tcp=");
        else if (has("--ecnK="))
            ecn_k = std::stoi(val("--ecnK="));
        else if (has("--queue="))
            queue = std::stoi(val("--queue="));
        else if (has("--topo="))
            topo = val("--topo=");
        else if (has("--topofile="))
            topofile = val("--topofile=");
        else if (has("--fail="))
            fail_spec = val("--fail=");
        else if (has("--leaves="))
            leaves = std::stoi(val("--leaves="));
        else if (has("--spines="))
            spines = std::stoi(val("--spines="));
        else if (has("--hpl="))
            hpl = std::stoi(val("--hpl="));
        else if (has("--fin="))
            fin = std::stoi(val("--fin="));
        else if (has("--spray="))
            spray = std::stoi(val("--spray="));
        else if (has("--RngSeed="))
            seed = std::stoll(val("--RngSeed="));
        else if (has("--RngRun="))
            run = std::stoll(val("--RngRun="));
        else if (has("--worlds="))
            worlds_file = val("--worlds=");
        else if (has("--ecmp_from="))
            ecmp_from = val("--ecmp_from=");
        else if (has("--hash_check="))
            hash_check = std::stoi(val("--hash_check="));
        else if (has("--max_slots="))
            max_slots = std::stoll(val("--max_slots="));
        else if (has("--host_lanes="))
            host_lanes = std::stoi(val("--host_lanes="));
        else if (has("--hbm_budget_gb="))
            budget_gb = std::stod(val("--hbm_budget_gb="));
        else if (has("--qtrace="))
            qtrace_file = val("--qtrace=");
        else if (has("--qtrace_from="))
            qtrace_from = std::stoll(val("--qtrace_from="));
        else if (has("--qtrace_until="))
            qtrace_until = std::stoll(val("--qtrace_until="));
        else if (a == "--general" || has("--ooo_segs=") || has("--rtt_ring=") || has("--graph_k="))
            ; // the reference's tuning flags: this build sizes its rings itself
        else
        {
            fprintf(stderr, "unknown argument %s\n", a.c_str());
            return 1;
        }
    }
    if (!qtrace_file.empty() && !tb_has_qtrace())
    {
        // the trace build, beside this program
        char self[4096];
        ssize_t n = readlink("/proc/self/exe", self, sizeof self - 1);
        std::string path = n > 0 ? std::string(self, n) : std::string(argv[0]);
        path = path.substr(0, path.find_last_of('/') + 1) + "twins-trace";
        execv(path.c_str(), argv);
        fprintf(stderr, "twins: --qtrace needs %s\n", path.c_str());
        return 1;
    }
    // the topology
    tb_topology T;
    memset(&T, 0, sizeof T);
    std::vector<int> la, lb, fa, fb, fu;
    std::vector<long long> ft;
    if (topo == "graph")
    {
        std::ifstream in(topofile);
        if (!in)
        {
            fprintf(stderr, "cannot open %s\n", topofile.c_str());
            return 1;
        }
        T.kind = TB_TOPO_GRAPH;
        std::string key;
        auto node = [](const std::string &x) { return x[0] == 'h' ? std::stoi(x.substr(1)) : -1 - std::stoi(x.substr(1)); };
        while (in >> key)
        {
            if (key == "hosts")
                in >> T.n_hosts;
            else if (key == "switches")
                in >> T.n_switches;
            else if (key == "link")
            {
                std::string a, b;
                in >> a >> b;
                la.push_back(node(a));
                lb.push_back(node(b));
            }
            else
                std::getline(in, key);
        }
        std::stringstream fs(fail_spec);
        for (std::string item; std::getline(fs, item, ',');)
        {
            if (item.empty())
                continue;
            std::vector<std::string> v;
            std::stringstream is(item);
            for (std::string x; std::getline(is, x, ':');)
                v.push_back(x);
            if (v.size() < 3)
            {
                fprintf(stderr, "--fail: T:sA:sB[:up]\n");
                return 1;
            }
            ft.push_back(std::stoll(v[0]));
            fa.push_back(std::stoi(v[1].substr(1)));
            fb.push_back(std::stoi(v[2].substr(1)));
            fu.push_back(v.size() > 3 && v[3] == "up");
        }
        T.n_links = (int)la.size();
        T.link_a = la.data();
        T.link_b = lb.data();
        T.n_fails = (int)ft.size();
        T.fail_t_ns = ft.data();
        T.fail_a = fa.data();
        T.fail_b = fb.data();
        T.fail_up = fu.data();
    }
    else if (topo == "leafspine")
    {
        T.kind = TB_TOPO_LEAFSPINE;
        T.leaves = leaves;
        T.spines = spines;
        T.hpl = hpl;
    }
    else if (topo == "fattree")
    {
        T.kind = TB_TOPO_FATTREE;
        T.k = k;
    }
    else
    {
        fprintf(stderr, "--topo: fattree, leafspine or graph\n");
        return 1;
    }
    if (!fail_spec.empty() && topo != "graph")
    {
        fprintf(stderr, "--fail needs --topo=graph\n");
        return 1;
    }
    const int H = T.kind == TB_TOPO_GRAPH ? T.n_hosts : T.kind == TB_TOPO_LEAFSPINE ? leaves * hpl : k * k * k / 4;
    if (tcp_of(tcp) < 0 || (flow_file.empty() && worlds_file.empty()) || H < 1)
    {
        fprintf(stderr, "usage: twins (--k=<4..32> | --topo=leafspine --leaves=L --spines=S --hpl=N | --topo=graph --topofile=F)\n"
                        "         (--flows=<csv> [--out=csv] [--tcp=dctcp|newreno|cubic] [--ecnK=30] [--queue=200] [--fin=0|1]\n"
                        "          [--ecmp_from=csv [--hash_check=1]] [--spray=1 [--RngSeed=1 --RngRun=1]]\n"
                        "          | --worlds=<file>: one world per line, flows=..,tcp=..,ecnK=..,queue=..,fin=..,ecmp_from=..,out=..)\n");
        return 1;
    }
    std::vector<World> worlds;
    if (worlds_file.empty())
        worlds.push_back({flow_file, ecmp_from, out, tcp_of(tcp), ecn_k, queue, fin});
    else
    {
        std::ifstream in(worlds_file);
        if (!in)
        {
            fprintf(stderr, "cannot open %s\n", worlds_file.c_str());
            return 1;
        }
        for (std::string line; std::getline(in, line);)
        {
            if (line.empty() || line[0] == '#')
                continue;
            World w{"", "", "", tcp_of(tcp), ecn_k, queue, fin};
            std::stringstream ss(line);
            for (std::string kv; std::getline(ss, kv, ',');)
            {
                size_t e = kv.find('=');
                std::string key = kv.substr(0, e), v = e == std::string::npos ? "" : kv.substr(e + 1);
                if (key == "flows")
                    w.flows = v;
                else if (key == "tcp" && tcp_of(v) >= 0)
                    w.tcp = tcp_of(v);
                else if (key == "ecnK")
                    w.ecn_k = std::stoi(v);
                else if (key == "queue")
                    w.queue = std::stoi(v);
                else if (key == "fin")
                    w.fin = std::stoi(v);
                else if (key == "ecmp_from")
                    w.ecmp_from = v;
                else if (key == "out")
                    w.out = v;
                else
                {
                    fprintf(stderr, "%s: bad entry %s\n", worlds_file.c_str(), kv.c_str());
                    return 1;
                }
            }
            if (w.flows.empty() || w.out.empty())
            {
                fprintf(stderr, "%s: every world needs flows= and out=\n", worlds_file.c_str());
                return 1;
            }
            worlds.push_back(w);
        }
    }
    tb_ctx *ctx = nullptr;
    if (tb_ctx_create(0, (unsigned long long)(budget_gb * 1e9), &ctx) != TB_OK)
    {
        fprintf(stderr, "twins: %s\n", tb_last_error());
        return 1;
    }
    if (host_lanes > 0)
        tb_set_launch(ctx, host_lanes, 0); // (else the launch shape is autotuned)
    if (!qtrace_file.empty() && tb_set_qtrace(ctx, 20000000, qtrace_from, qtrace_until) != TB_OK)
    {
        fprintf(stderr, "twins: %s\n", tb_last_error());
        return 1;
    }
    std::vector<Flows> flows(worlds.size());
    int hash_same = 0, hash_n = 0;
    for (size_t w = 0; w < worlds.size(); w++)
    {
        if (!load_flows(worlds[w].flows, H, flows[w]))
        {
            fprintf(stderr, "cannot open %s\n", worlds[w].flows.c_str());
            return 1;
        }
        Flows &f = flows[w];
        std::vector<unsigned> hd, ha;
        if (!worlds[w].ecmp_from.empty() && !load_hashes(worlds[w].ecmp_from, f.src.size(), hd, ha))
        {
            fprintf(stderr, "%s has no hash columns for every flow\n", worlds[w].ecmp_from.c_str());
            return 1;
        }
        tb_tcp_params p{worlds[w].tcp, worlds[w].ecn_k, worlds[w].queue, worlds[w].fin, spray, (unsigned)seed, (unsigned long long)run};
        int id = 0;
        int r = tb_world_add_tcp(ctx, &T, (int)f.src.size(), f.src.data(), f.dst.data(), f.size.data(), f.start.data(), f.conn.data(),
                                 hash_check || hd.empty() ? nullptr : hd.data(), hash_check || ha.empty() ? nullptr : ha.data(), &p, &id);
        if (r != TB_OK)
        {
            fprintf(stderr, "%s: %s\n", worlds[w].flows.c_str(), tb_last_error());
            return 1;
        }
        if (hash_check && !hd.empty())
        {
            std::vector<unsigned> md(f.src.size()), ma(f.src.size());
            tb_hashes(ctx, id, md.data(), ma.data());
            std::vector<char> first(f.src.size(), 1);
            std::vector<long long> seen;
            for (size_t i = 0; i < f.src.size(); i++)
            {
                if (f.conn[i] >= 0)
                {
                    bool dup = false;
                    for (long long c : seen)
                        dup |= c == f.conn[i];
                    if (dup)
                        continue;
                    seen.push_back(f.conn[i]);
                }
                hash_n++;
                hash_same += md[i] == hd[i] && ma[i] == ha[i];
            }
        }
    }
    if (hash_check)
    {
        printf("ECMP hashes: %d of %d connections as ns-3's\n", hash_same, hash_n);
        tb_ctx_destroy(ctx);
        return hash_same == hash_n ? 0 : 1;
    }
    int r = tb_run(ctx, max_slots);
    if (r < 0)
    {
        fprintf(stderr, "twins: %s\n", tb_last_error());
        tb_ctx_destroy(ctx);
        return 1;
    }
    tb_stats st;
    tb_get_stats(ctx, &st);
    unsigned long long tot[16] = {0};
    long long done_total = 0, total = 0;
    for (size_t w = 0; w < worlds.size(); w++)
    {
        Flows &f = flows[w];
        std::vector<long long> est(f.src.size()), done(f.src.size());
        tb_results(ctx, (int)w, est.data(), done.data());
        unsigned long long ev[16];
        tb_counters(ctx, (int)w, ev, 16);
        for (int i = 0; i < 16; i++)
            tot[i] += ev[i];
        std::ofstream o(worlds[w].out);
        o << "src,dst,flow_size,start_ns,established_ns,completed_ns\n";
        for (size_t i = 0; i < f.src.size(); i++)
        {
            o << f.src[i] << "," << f.dst[i] << "," << f.size[i] << "," << f.start[i] << "," << est[i] << "," << done[i] << "\n";
            total++;
            done_total += done[i] >= 0;
        }
    }
    printf("Simulation Duration: %.6fs\n", st.kernel_ms / 1000.0);
    printf("Executed Slots: %lld\n", st.slots);
    printf("flows %lld completed %lld wall %.4f s drops %llu marks %llu retx %llu rto %llu | packet-events %llu (hosts %llu, switch "
           "ports %llu) slots-run %lld launches %lld | overflow: active %llu due %llu ring %llu ooo %llu tx-cap %llu | "
           "undecided-ties %llu\n",
           total, done_total, st.kernel_ms / 1000.0, tot[0], tot[1], tot[2], tot[3], st.packet_events, st.host_events, st.switch_events,
           st.slots_run, st.launches, tot[7], tot[8], tot[9], tot[10], tot[11], tot[4]);
    if (r == TB_WARN_INEXACT)
        fprintf(stderr, "warning: a capacity overflowed; the results may differ from the reference\n");
    if (!qtrace_file.empty())
    {
        unsigned long long n = 0;
        tb_qtrace(ctx, nullptr, 0, &n);
        std::vector<tb_qrec> q(n);
        tb_qtrace(ctx, q.data(), n, &n);
        std::stable_sort(q.begin(), q.end(), [](const tb_qrec &a, const tb_qrec &b) {
            if (a.ts != b.ts)
                return a.ts < b.ts;
            if (a.node != b.node)
                return a.node < b.node;
            return a.dev < b.dev;
        });
        FILE *o = fopen(qtrace_file.c_str(), "w");
        if (!o)
        {
            fprintf(stderr, "cannot write %s\n", qtrace_file.c_str());
            return 1;
        }
        for (const tb_qrec &x : q)
        {
            // data, SYN-ACK, SYN, else an ACK (FIN, FIN-ACK and pure ACKs)
            const char *kind = (x.flags & 32) ? "D" : (x.flags & 2) ? ((x.flags & 1) ? "SA" : "S") : "A";
            fprintf(o, "%lld %d %d %d %d %s %u %d\n", x.ts, x.node, x.dev, x.src, x.dst, kind, x.sa, (int)x.qlen);
        }
        fclose(o);
        printf("qtrace: %llu records\n", n);
    }
    if (worlds.size() > 1)
        printf("worlds %zu\n", worlds.size());
    tb_ctx_destroy(ctx);
    return 0;
}
