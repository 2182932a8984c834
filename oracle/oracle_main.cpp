// TEST INFRASTRUCTURE — the oracle's command line. It takes the reference twins' flags
// (src/main.cu:155-222) for one world and writes the same fct.csv (src/main.cu:1143-1153):
//   twins_oracle (--k=K | --topo=leafspine --leaves=L --spines=S --hpl=N | --topo=graph --topofile=F
//                 [--fail=T:sA:sB[:up],...]) --flows=CSV [--out=CSV] [--tcp=dctcp|newreno|cubic]
//                [--ecnK=30] [--queue=200] [--fin=0|1] [--spray=0|1 --RngSeed=1 --RngRun=1]
//                [--ecmp_from=CSV] [--max_slots=N] [--chain_runs=9|25] [--hash_out=CSV]
// The last line printed is a summary with the packet-event count and the event-loop time.
#include <chrono>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>

#include "tcp_oracle.h"

using namespace oracle;

static bool read_hashes(const std::string &path, size_t n, WorldSpec &w)
{
    std::ifstream in(path);
    if (!in)
        return false;
    std::string line;
    std::getline(in, line);
    w.hash_data.assign(n, 0);
    w.hash_ack.assign(n, 0);
    size_t i = 0;
    while (i < n && std::getline(in, line))
    {
        std::vector<std::string> v;
        std::stringstream ss(line);
        for (std::string f; std::getline(ss, f, ',');)
            v.push_back(f);
        if (v.size() < 8)
            return false;
        w.hash_data[i] = (uint32_t)std::stoul(v[6]);
        w.hash_ack[i] = (uint32_t)std::stoul(v[7]);
        i++;
    }
    w.have_hashes = i == n;
    return w.have_hashes;
}

int main(int argc, char **argv)
{
    WorldSpec w;
    std::string flows, out = "fct.csv", tcp = "dctcp", topo = "fattree", topofile, fail, ecmp_from, hash_out;
    for (int i = 1; i < argc; i++)
    {
        std::string a = argv[i];
        auto has = [&](const char *p) { return a.rfind(p, 0) == 0; };
        auto val = [&](const char *p) { return a.substr(strlen(p)); };
        if (has("--k="))
            w.topo.k = std::stoi(val("--k="));
        else if (has("--flows="))
            flows = val("--flows=");
        else if (has("--out="))
            out = val("--out=");
        else if (has("--tcp="))
            tcp = val("--tcp=");
        else if (has("--ecnK="))
            w.red_k = std::stoi(val("--ecnK="));
        else if (has("--queue="))
            w.qcap = std::stoi(val("--queue="));
        else if (has("--topo="))
            topo = val("--topo=");
        else if (has("--topofile="))
            topofile = val("--topofile=");
        else if (has("--fail="))
            fail = val("--fail=");
        else if (has("--leaves="))
            w.topo.leaves = std::stoi(val("--leaves="));
        else if (has("--spines="))
            w.topo.spines = std::stoi(val("--spines="));
        else if (has("--hpl="))
            w.topo.hpl = std::stoi(val("--hpl="));
        else if (has("--fin="))
            w.fin = std::stoi(val("--fin=")) != 0;
        else if (has("--spray="))
            w.spray = std::stoi(val("--spray=")) != 0;
        else if (has("--RngSeed="))
            w.rng_seed = (uint32_t)std::stoll(val("--RngSeed="));
        else if (has("--RngRun="))
            w.rng_run = (uint64_t)std::stoll(val("--RngRun="));
        else if (has("--max_slots="))
            w.max_slots = std::stoll(val("--max_slots="));
        else if (has("--chain_runs="))
            w.chain_runs = std::stoi(val("--chain_runs="));
        else if (has("--ecmp_from="))
            ecmp_from = val("--ecmp_from=");
        else if (has("--hash_out="))
            hash_out = val("--hash_out=");
        else if (a == "--general" || has("--host_lanes=") || has("--ooo_segs=") || has("--rtt_ring=") || has("--graph_k="))
            ; // the reference's tuning flags: no effect on results
        else
        {
            fprintf(stderr, "unknown argument %s\n", a.c_str());
            return 1;
        }
    }
    w.cc = tcp == "newreno" ? CC_NEWRENO : tcp == "cubic" ? CC_CUBIC : CC_DCTCP;
    if (tcp != "dctcp" && tcp != "newreno" && tcp != "cubic")
    {
        fprintf(stderr, "--tcp: dctcp, newreno or cubic\n");
        return 1;
    }
    if (w.chain_runs < 1 || w.chain_runs > 25)
    {
        fprintf(stderr, "--chain_runs: 1..25\n");
        return 1;
    }
    std::string err;
    if (topo == "graph")
    {
        if (!load_topofile(topofile, w.topo, err) || !parse_fail_spec(fail, w.topo, err))
        {
            fprintf(stderr, "%s\n", err.c_str());
            return 1;
        }
    }
    else if (topo == "leafspine")
        w.topo.kind = TOPO_LEAFSPINE;
    else if (topo != "fattree" || w.topo.k < 4 || (w.topo.k & (w.topo.k - 1)))
    {
        fprintf(stderr, "bad topology\n");
        return 1;
    }
    if (flows.empty())
    {
        fprintf(stderr, "--flows is required\n");
        return 1;
    }
    w.flows = load_flows(flows, hosts_of(w.topo));
    if (!ecmp_from.empty() && !read_hashes(ecmp_from, w.flows.size(), w))
    {
        fprintf(stderr, "%s: no hash columns for every flow\n", ecmp_from.c_str());
        return 1;
    }
    auto t0 = std::chrono::steady_clock::now();
    WorldResult r = run_world(w);
    double sec = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    if (r.slots < 0)
        return 1;
    {
        std::ofstream o(out);
        o << "src,dst,flow_size,start_ns,established_ns,completed_ns\n";
        for (size_t i = 0; i < w.flows.size(); i++)
            o << w.flows[i].src << "," << w.flows[i].dst << "," << w.flows[i].size << "," << w.flows[i].start_ns << ","
              << r.est_ns[i] << "," << r.done_ns[i] << "\n";
    }
    if (!hash_out.empty())
    {
        std::ofstream o(hash_out);
        o << "hash_data,hash_ack\n";
        for (size_t i = 0; i < w.flows.size(); i++)
            o << r.hash_data[i] << "," << r.hash_ack[i] << "\n";
    }
    printf("oracle: flows %zu completed %u slots %lld slots_run %lld events %llu host_events %llu switch_events %llu "
           "drops %llu marks %llu retx %llu rto %llu undecided-ties %llu seconds %.6f\n",
           w.flows.size(), r.completed, (long long)r.slots, (long long)r.slots_run, (unsigned long long)r.events,
           (unsigned long long)r.host_events, (unsigned long long)r.switch_events, (unsigned long long)r.drops,
           (unsigned long long)r.marks, (unsigned long long)r.retx, (unsigned long long)r.rtos,
           (unsigned long long)r.ties, sec);
    return 0;
}
